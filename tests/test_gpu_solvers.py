"""The optional level-loop solvers (VFB_SOLVER=coop: one cooperative
persistent kernel with a bounded grid barrier between phases; cluster: one
instance per thread-block cluster, large levels promoted to the graph solver)
run the same phases as the default graph solver, so their results equal the
oracle's (LTL_BS.cu:1069-1532 restated): exact and relaxed keys, planted
instances, levels whose first solution is a unary candidate, and relaxed-key
collisions that make a level be built again in full."""
import pytest

import oracle
import vfb_b200
from vfb_b200 import synth
from tests import cases

pytestmark = pytest.mark.gpu


def _instances():
    insts = cases.small_exact_cases()[:6] + cases.relaxed_cases(3)[:3] + cases.planted_cases(4)
    insts += cases.mirrored_cases(count=4)
    insts.append(synth.config_planted())
    return insts


@pytest.fixture(scope="module")
def expected():
    insts = _instances()
    return insts, [oracle.solve(oracle.Problem.from_instance(i)) for i in insts]


def _same(got, ref):
    return (got.rpn == ref["rpn"] and got.level_rows == ref["level_rows"]
            and got.level_cands == ref["level_cands"])


@pytest.mark.parametrize("solver", ["coop", "cluster"])
def test_optional_solver_matches_oracle(monkeypatch, expected, solver):
    monkeypatch.setenv("VFB_SOLVER", solver)
    insts, refs = expected
    probs = [vfb_b200.Problem.from_instance(i) for i in insts]
    with vfb_b200.Engine() as eng:
        solo = [eng.solve(p) for p in probs]
        batch = eng.batch_solve(probs)
    bad = [i.name for i, g, r in zip(insts, solo, refs) if not _same(g, r)]
    assert not bad, bad
    bad = [i.name for i, g, r in zip(insts, batch, refs) if not _same(g, r)]
    assert not bad, bad
