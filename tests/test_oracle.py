"""CPU checks of the oracle (the checker of the GPU path) and of the word
identities the kernels rely on.  No GPU needed."""
import random

import pytest

import oracle
from vfb_b200 import synth
from tests import cases

M64 = (1 << 64) - 1


def _doubling_until(l, r):
    # LTL_BS.cu:222-233 / ltl_nocache.cu:136-148
    for s in (1, 2, 4, 8, 16):
        r |= l & (r >> s)
        l &= l >> s
    return r | (l & (r >> 32))


def _brev(x):
    return int(f"{x:064b}"[::-1], 2)


def _carry_until(l, r):
    # the kernels' form: bit-reverse, one addition as a carry chain
    lr, rr = _brev(l), _brev(r)
    a = lr | rr
    s = (a + rr) & M64
    c = s ^ a ^ rr
    cout = 1 if s < a else 0
    return _brev(((c >> 1) | (cout << 63)) & M64)


def _doubling_finally(w):
    for s in (1, 2, 4, 8, 16, 32):
        w |= w >> s
    return w


def _clz_finally(w):
    return 0 if w == 0 else (M64 >> (64 - w.bit_length()))


def test_until_carry_form_equals_doubling():
    rng = random.Random(7)
    words = [0, M64, 1, 1 << 63, 0xAAAAAAAAAAAAAAAA, 0x5555555555555555]
    words += [rng.getrandbits(64) for _ in range(300)]
    words += [rng.getrandbits(64) & rng.getrandbits(64) & rng.getrandbits(64) for _ in range(200)]
    for l in words[:120]:
        for r in words[:60] + [rng.getrandbits(64) for _ in range(20)]:
            assert _carry_until(l, r) == _doubling_until(l, r)


def test_finally_clz_form_equals_doubling():
    rng = random.Random(8)
    for w in [0, 1, M64, 1 << 63] + [rng.getrandbits(rng.randint(1, 64)) for _ in range(2000)]:
        assert _clz_finally(w) == _doubling_finally(w)


def test_oracle_operator_semantics_match_python_evaluator():
    inst = cases.random_instance(11, 3, 3, 3, [5, 7, 9, 11, 13, 64], 5)
    prob = oracle.Problem.from_instance(inst)
    atoms = inst.atom_words()
    lens = inst.lengths()
    for op in "~XFG":
        got = oracle.apply(prob, op, atoms[0])
        exp = [synth.eval_rpn_word([0, op], [atoms[0][i]], lens[i]) for i in range(len(lens))]
        assert got == exp
    for op in "&|U":
        got = oracle.apply(prob, op, atoms[1], atoms[2])
        exp = [synth.eval_rpn_word([0, 1, op], [atoms[1][i], atoms[2][i]], lens[i])
               for i in range(len(lens))]
        assert got == exp


def test_exact_key_packs_bits_trace_major():
    # three traces of lengths 4, 3, 5 -> 12 bits, trace 0 in bits 0..3
    inst = cases.random_instance(1, 1, 1, 2, [4, 3, 5], 3)
    prob = oracle.Problem.from_instance(inst)
    cs = [0b1011, 0b110, 0b10001]
    h, l = oracle.make_key(prob, cs)
    assert h == 0
    assert l == 0b1011 | (0b110 << 4) | (0b10001 << 7)


def test_exact_key_spans_two_words():
    # 2 traces of length 63 + 1 of 0.. -> bits 63..125 land in h
    inst = cases.random_instance(2, 1, 1, 1, [63, 63], 3)
    prob = oracle.Problem.from_instance(inst)
    a = (1 << 63) - 1
    h, l = oracle.make_key(prob, [a, 5])
    assert l == a and h == 5


def test_hash_key_xor_fold_halves():
    inst = cases.random_instance(3, 1, 3, 3, 32, 3)   # 192 bits > 126 -> type 3
    prob = oracle.Problem.from_instance(inst)

    def fin(x):
        x = ((x ^ (x >> 30)) * 0xBF58476D1CE4E5B9) & M64
        x = ((x ^ (x >> 27)) * 0x94D049BB133111EB) & M64
        return x ^ (x >> 31)

    cs = [3, 5, 7, 11, 13, 17]
    h, l = oracle.make_key(prob, cs)
    eh = fin(3) ^ fin(5) ^ fin(7)
    el = fin(11) ^ fin(13) ^ fin(17)
    assert (h, l) == (eh if eh != M64 else M64 - 1, el if el != M64 else M64 - 1)


def test_sampled_and_prefix_keys():
    lens = [40, 40, 40, 40]                      # S = 160 > 126
    inst = cases.random_instance(4, 1, 2, 2, lens, 3, rlx_type=1)
    prob = oracle.Problem.from_instance(inst)
    cs = [(1 << 40) - 1, 0, (1 << 40) - 1, 0]
    h, l = oracle.make_key(prob, cs)
    # stride 160//126 = 1: bits 0..125 are trace 0, trace 1, then 46 bits of trace 2
    assert l == (1 << 40) - 1
    assert h == ((1 << 40) - 1) << (80 - 63)
    inst2 = cases.random_instance(4, 1, 2, 2, lens, 3, rlx_type=2)
    prob2 = oracle.Problem.from_instance(inst2)
    # type 2 keeps (126*40+160)//160 = 32 bits of each trace
    h2, l2 = oracle.make_key(prob2, [M64 >> 24, 0, 0, 0])
    assert l2 == (1 << 32) - 1 and h2 == 0


def test_small_config_solution():
    inst = synth.config_small()
    res = oracle.solve(oracle.Problem.from_instance(inst))
    assert res["status"] == oracle.FOUND
    ok, _ = oracle.eval_rpn(oracle.Problem.from_instance(inst), res["rpn"])
    assert ok == 1


@pytest.mark.parametrize("inst", cases.small_exact_cases(), ids=lambda i: i.name)
def test_cached_search_equals_exhaustive_numbering(inst):
    """In exact mode the cached, deduplicated search returns the first formula
    of the exhaustive ltl_nocache numbering (same size, same formula)."""
    prob = oracle.Problem.from_instance(inst)
    cached = oracle.solve(prob)
    exh = oracle.exhaustive(prob, 1 << 24)
    if exh["status"] == oracle.LIMIT:
        pytest.skip("exhaustive budget")
    assert cached["status"] == exh["status"]
    if exh["status"] == oracle.FOUND:
        assert cached["size"] == exh["size"]
        assert cached["rpn"] == exh["rpn"]


@pytest.mark.parametrize("inst", cases.planted_cases(), ids=lambda i: i.name)
def test_planted_size_bounds_result(inst):
    prob = oracle.Problem.from_instance(inst)
    res = oracle.solve(prob)
    assert res["status"] == oracle.FOUND
    assert res["size"] <= len(inst.planted)
    ok, _ = oracle.eval_rpn(prob, res["rpn"])
    assert ok == 1
    assert len(res["rpn"]) == res["size"]


@pytest.mark.parametrize("rlx", [1, 2, 3])
def test_parallel_port_equals_scalar(rlx):
    for inst in cases.relaxed_cases(rlx) + cases.planted_cases(3):
        a = oracle.solve(oracle.Problem.from_instance(inst, threads=1, rlx_type=rlx))
        b = oracle.solve(oracle.Problem.from_instance(inst, threads=4, rlx_type=rlx))
        assert a["status"] == b["status"]
        assert a["rpn"] == b["rpn"]
        assert a["level_rows"] == b["level_rows"]
        assert a["level_cands"] == b["level_cands"]


def test_refcompat_drops_odd_until_pairs():
    """The reference's U launch evaluates only even pair indices (LTL_BS.cu:397-403)."""
    inst = synth.config_small()
    can = oracle.solve(oracle.Problem.from_instance(inst, max_size=10))
    ref = oracle.solve(oracle.Problem.from_instance(inst, mode=oracle.REFCOMPAT))
    assert ref["status"] == can["status"]
    # level 2 has no binary operator: identical
    assert ref["level_rows"][:2] == can["level_rows"][:2]


def test_refcompat_level3_candidates():
    inst = cases.random_instance(77, 3, 3, 3, 6, 3)
    # force "not found" by labelling identical traces: pos 0 == neg 0
    inst.neg[0] = inst.pos[0]
    can = oracle.solve(oracle.Problem.from_instance(inst))
    ref = oracle.solve(oracle.Problem.from_instance(inst, mode=oracle.REFCOMPAT))
    assert can["status"] == ref["status"] == oracle.NOT_FOUND
    n1, n2 = can["level_rows"][0], can["level_rows"][1]
    # canonical level 3: ~,X,F,G of level 2, & and | over level1 x level1, U over level1 x level1
    assert can["level_cands"][2] == 4 * n2 + 3 * n1 * n1
    # LTL_BS: U covers even pairs of level1 x level1, both orientations
    assert ref["level_cands"][2] == 4 * n2 + 2 * n1 * n1 + 2 * ((n1 * n1 + 1) // 2)


def test_bs_stage_returns_solutions():
    # the BS stage's formulas are solutions, larger than the search's max size
    from tests import cases as _cases
    found = 0
    for seed in range(8000, 8010):
        inst = _cases.random_instance(seed, 3, 4, 4, [5, 6, 7, 8, 5, 6, 7, 8], 3)
        p = oracle.Problem.from_instance(inst)
        if oracle.solve(p)["status"] != oracle.NOT_FOUND:
            continue
        r = oracle.solve_bs(p, 8)
        if r["status"] == oracle.FOUND:
            found += 1
            assert r["size"] > 3 and len(r["rpn"]) == r["size"]
            assert oracle.eval_rpn(p, r["rpn"])[0] == 1
            assert set(t for t in r["rpn"] if isinstance(t, str)) <= {"~", "&", "|", "X", "F", "G", "U"}
    assert found >= 3
