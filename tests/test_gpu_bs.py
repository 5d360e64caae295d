"""BS stage (vfb_solve_bs) against the oracle's restatement."""
import pytest

import oracle
import vfb_b200
from tests import cases

pytestmark = pytest.mark.gpu

# (seed, max size, BS max size): the search to max size finds nothing and the
# BS stage finds a combination of size 5..8
FOUND = [(8000, 3, 8), (8001, 3, 8), (8005, 3, 8), (8006, 3, 8)]


def _inst(seed, max_size):
    return cases.random_instance(seed, 3, 4, 4, [5, 6, 7, 8, 5, 6, 7, 8], max_size)


def _check(engine, inst, bs_max):
    got = engine.solve_bs(vfb_b200.Problem.from_instance(inst), bs_max)
    want = oracle.solve_bs(oracle.Problem.from_instance(inst), bs_max)
    status = {oracle.FOUND: vfb_b200.OK, oracle.NOT_FOUND: vfb_b200.NOT_FOUND}[want["status"]]
    assert got.status == status
    assert got.size == want["size"]
    assert got.level_rows == want["level_rows"]
    assert got.level_cands == want["level_cands"]
    assert got.total_rows == want["total_rows"]
    if got.status == vfb_b200.OK:
        assert got.rpn == want["rpn"]
        assert got.solution_index == want["solution_index"]
        ok, _ = oracle.eval_rpn(oracle.Problem.from_instance(inst), got.rpn)
        assert ok == 1
    return got


@pytest.mark.parametrize("seed,max_size,bs_max", FOUND)
def test_bs_equals_oracle(engine, seed, max_size, bs_max):
    got = _check(engine, _inst(seed, max_size), bs_max)
    assert got.status == vfb_b200.OK and got.size > max_size


def test_bs_not_found(engine):
    inst = cases.random_instance(4242, 2, 3, 3, 5, 3)
    inst.neg[0] = inst.pos[0]          # contradictory sample
    got = _check(engine, inst, 7)
    assert got.status == vfb_b200.NOT_FOUND


def test_bs_not_needed(engine):
    # the search itself succeeds: the BS stage does not run
    inst = _inst(8000, 8)
    got = engine.solve_bs(vfb_b200.Problem.from_instance(inst), 10)
    solo = engine.solve(vfb_b200.Problem.from_instance(inst))
    assert (got.status, got.size, got.rpn, got.level_rows) == (solo.status, solo.size, solo.rpn, solo.level_rows)


def test_bs_relaxed_keys(engine):
    # the search uses relaxed keys (more than 126 trace bits); the BS vectors are exact
    for seed in range(8100, 8130):
        inst = cases.random_instance(seed, 3, 6, 6, 24, 3)
        want = oracle.solve_bs(oracle.Problem.from_instance(inst), 7)
        if want["status"] == oracle.FOUND and want["size"] > 3:
            _check(engine, inst, 7)
            return
    pytest.skip("no seed in range needs the BS stage")
