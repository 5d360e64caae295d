"""The native instance generator (vfb_synth_planted) draws exactly the Python
generator's random stream: same instances for the same seeds."""
import pytest

from vfb_b200 import synth


@pytest.mark.parametrize("seed", [1, 5, 17])
def test_native_equals_python(seed):
    for lengths, a, size, npos, nneg, p in [((4, 64), 3, 7, 9, 10, 0.5), (16, 4, 9, 20, 20, 0.5),
                                            ((3, 10), 2, 4, 3, 2, 0.3)]:
        r1, r2 = synth.Rng(seed), synth.Rng(seed)
        a1 = synth.planted_instance(r1, a, size, npos, nneg, lengths, p, size + 2, native=True)
        a2 = synth.planted_instance(r2, a, size, npos, nneg, lengths, p, size + 2, native=False)
        assert (a1.pos, a1.neg, a1.planted) == (a2.pos, a2.neg, a2.planted)
        assert r1.s == r2.s


def test_configs_are_stable():
    c2 = synth.config_planted()
    assert c2.num_vars == 4 and len(c2.pos) == 20 and len(c2.neg) == 20
    assert synth.rpn_to_infix(c2.planted, c2.names) == "X((a2) | (~(X((G(a2)) U (a1)))))"
    batch = synth.config_batch(count=8)
    assert len(batch) == 8 and all(2 <= b.num_vars <= 8 for b in batch)


def test_large_deep_seed_rule():
    """The deep large instance is the first seed from 2 on whose large-shape
    instance has no formula of size 9 or less: every seed before it is solved
    by the oracle within size 9 (seed 2, the shape's own seed, by a single
    proposition)."""
    import os

    import oracle
    sizes = {}
    for seed in range(2, synth.LARGE_DEEP_SEED):
        inst = synth.config_large(seed, max_size=9)
        r = oracle.solve(oracle.Problem.from_instance(inst, threads=os.cpu_count() or 1))
        assert r["status"] == oracle.FOUND, (seed, r["status"])
        sizes[seed] = r["size"]
    assert sizes[2] == 1
    assert max(sizes.values()) <= 9
