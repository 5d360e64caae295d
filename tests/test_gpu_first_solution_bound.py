"""Levels whose first solution is a unary candidate (~ X F G over the level
below).  The rows of every stored level record, when they are written, which
of their ~ X F G candidates satisfy the sample; the next level's plan starts
its search with that candidate as the bound on the first solution, and the
size splits run before the unary group.  These instances, picked by the
oracle (LTL_BS.cu:1069-1532 restated) for a solution whose top operator is
unary, check that the result still equals the oracle's: formula, solution
index and every level's rows and candidates, with the default launch shape
and with one CTA taking the tiles in order.
"""
import pytest

import oracle
import vfb_b200
from vfb_b200 import synth

pytestmark = pytest.mark.gpu


def _unary_top_instances(want: int = 12):
    out, tops = [], set()
    for s in range(2000):
        rng = synth.Rng(7100 + s)
        a = 2 + rng.below(5)
        size = 5 + rng.below(6)
        t = 10 + rng.below(40)
        npos = 1 + rng.below(t - 1)
        inst = synth.planted_instance(rng, a, size, npos, t - npos, (2, 40), 0.4, size + 2,
                                      name=f"unary-top{s}")
        inst.rlx_type = 1 + s % 3
        ref = oracle.solve(oracle.Problem.from_instance(inst))
        if ref["status"] != oracle.FOUND or ref["size"] < 5 or ref["rpn"][-1] not in ("~", "X", "F", "G"):
            continue
        out.append((inst, ref))
        tops.add(ref["rpn"][-1])
        if len(out) >= want and len(tops) >= 3:
            break
    return out, tops


@pytest.fixture(scope="module")
def unary_top():
    cases, tops = _unary_top_instances()
    assert len(cases) >= 8 and len(tops) >= 3, (len(cases), tops)
    return cases


def _check(eng, cases):
    for inst, ref in cases:
        got = eng.solve(vfb_b200.Problem.from_instance(inst))
        assert got.status == vfb_b200.OK, inst.name
        assert got.rpn == ref["rpn"], inst.name
        assert got.solution_index == ref["solution_index"], inst.name
        assert got.level_rows == ref["level_rows"], inst.name
        assert got.level_cands == ref["level_cands"], inst.name


def test_unary_first_solution_default_shape(unary_top):
    with vfb_b200.Engine() as eng:
        _check(eng, unary_top)


def test_unary_first_solution_tiles_in_order(unary_top):
    with vfb_b200.Engine() as eng:
        eng.set_tune({"rows": [1] * vfb_b200.TUNE_BANDS, "tiles_log2": [16] * vfb_b200.TUNE_BANDS,
                      "blocks": [1] * vfb_b200.TUNE_BANDS})
        _check(eng, unary_top)


def test_unary_first_solution_in_a_batch(unary_top):
    probs = [vfb_b200.Problem.from_instance(inst) for inst, _ in unary_top]
    with vfb_b200.Engine() as eng:
        got = eng.batch_solve(probs)
    for r, (inst, ref) in zip(got, unary_top):
        assert (r.rpn, r.level_rows, r.level_cands) == (ref["rpn"], ref["level_rows"], ref["level_cands"]), \
            inst.name
