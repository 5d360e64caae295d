"""Operator costs (vfb_solve_costs) against the oracle's weighted order."""
import pytest

import oracle
import vfb_b200
from tests import cases
from vfb_b200 import synth

pytestmark = pytest.mark.gpu

WEIGHTS = [([1, 2, 2, 2, 1, 1, 1, 3], 1), ([2, 1, 3, 3, 2, 2, 2, 2], 2), ([1, 1, 2, 3, 1, 2, 2, 1], 1)]


def _check(engine, inst, costs, neg):
    got = engine.solve_costs(vfb_b200.Problem.from_instance(inst), costs, neg)
    want = oracle.solve(oracle.Problem.from_instance(inst, costs=costs, neg_type=neg))
    status = {oracle.FOUND: vfb_b200.OK, oracle.NOT_FOUND: vfb_b200.NOT_FOUND}[want["status"]]
    assert got.status == status
    assert got.size == want["size"]
    assert got.rpn == want["rpn"]
    assert got.level_rows == want["level_rows"]
    assert got.level_cands == want["level_cands"]
    if got.status == vfb_b200.OK:
        assert got.solution_index == want["solution_index"]
        ok, _ = oracle.eval_rpn(oracle.Problem.from_instance(inst), got.rpn)
        assert ok == 1
    return got


@pytest.mark.parametrize("costs,neg", WEIGHTS, ids=["w1", "w2", "w3"])
@pytest.mark.parametrize("seed", [9000, 9003, 9007, 9011])
def test_costs_exact_keys(engine, costs, neg, seed):
    _check(engine, cases.random_instance(seed, 2, 3, 3, [3, 4, 5, 3, 4, 5], 9), costs, neg)


@pytest.mark.parametrize("costs,neg", WEIGHTS, ids=["w1", "w2", "w3"])
def test_costs_relaxed_keys(engine, costs, neg):
    inst = cases.planted_cases(3)[2]
    inst.max_size = 9
    _check(engine, inst, costs, neg)


def test_unit_costs_equal_solve(engine):
    inst = synth.config_planted()
    a = engine.solve(vfb_b200.Problem.from_instance(inst))
    b = engine.solve_costs(vfb_b200.Problem.from_instance(inst), [1] * 8, 1)
    assert (a.status, a.size, a.rpn, a.level_rows, a.level_cands) == (b.status, b.size, b.rpn, b.level_rows,
                                                                        b.level_cands)
