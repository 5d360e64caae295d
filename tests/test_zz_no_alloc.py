"""vfb_solve_noalloc -- the solve for callers that cannot allocate.

Some callers may not allocate device memory while they run (their device heap
belongs to another allocator, or cudaMalloc's implicit synchronisation is not
acceptable in their loop).  vfb_solve_noalloc serves them from a static
device array; these tests call it through the C ABI and check it against
vfb_solve bit for bit, twice in a row (the array keeps the previous call's
contents, so the second call proves the reset), and check the clear VFB_OOM
refusal when a search outgrows the array.

This file is collected last so that a run stopping at the first failure has
already run every other test; it also passes when run alone.
"""
import pytest

import vfb_b200
from vfb_b200 import synth
from tests import cases

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def plain_engine():
    eng = vfb_b200.Engine()
    yield eng
    eng.close()


def _same(a, b):
    return (a.status, a.size, a.rpn, a.level_rows, a.level_cands, a.total_rows, a.solution_index) == \
           (b.status, b.size, b.rpn, b.level_rows, b.level_cands, b.total_rows, b.solution_index)


INSTANCES = ([synth.config_small(), synth.config_planted()] + cases.small_exact_cases()[1:5]
             + cases.relaxed_cases(1)[:1] + cases.relaxed_cases(2)[:1] + cases.relaxed_cases(3)[:2]
             + cases.planted_cases(4))


@pytest.mark.parametrize("inst", INSTANCES, ids=lambda i: i.name)
def test_noalloc_equals_solve_twice(plain_engine, inst):
    prob = vfb_b200.Problem.from_instance(inst)
    want = plain_engine.solve(prob)
    first = vfb_b200.solve_noalloc(prob)
    second = vfb_b200.solve_noalloc(prob)
    assert _same(first, want), (first, want)
    assert _same(second, want), (second, want)
    assert first.kernel_launches > 0


def test_noalloc_alternating_instances(plain_engine):
    """Back-to-back calls on different instances: each starts from a clean array."""
    a = vfb_b200.Problem.from_instance(synth.config_planted())
    b = vfb_b200.Problem.from_instance(cases.relaxed_cases(3)[0])
    wa, wb = plain_engine.solve(a), plain_engine.solve(b)
    for _ in range(2):
        assert _same(vfb_b200.solve_noalloc(a), wa)
        assert _same(vfb_b200.solve_noalloc(b), wb)


def test_noalloc_refuses_searches_larger_than_the_array():
    inst = cases.random_instance(4242, 4, 5, 5, 16, 9)
    inst.neg[0] = inst.pos[0]        # unsolvable: ~1e6 characteristic sets by size 9
    res = vfb_b200.solve_noalloc(vfb_b200.Problem.from_instance(inst))
    assert res.status == vfb_b200.OOM
    # the sizes finished before the array ran out are reported
    assert 1 <= res.size < 9
    assert res.level_rows[0] == 4
