"""Cache-free search (vfb_solve_exhaustive) against the oracle's exhaustive
enumerator and the reference's ltl_nocache runs."""
import os
import subprocess

import pytest

import oracle
import vfb_b200
from oracle import reference
from tests import cases
from tests.test_golden import RUNS, instance_from_json
from vfb_b200 import synth

pytestmark = pytest.mark.gpu


def _check(engine, inst):
    prob = vfb_b200.Problem.from_instance(inst)
    got = engine.solve_exhaustive(prob)
    want = oracle.exhaustive(oracle.Problem.from_instance(inst), 1 << 26)
    assert want["status"] in (oracle.FOUND, oracle.NOT_FOUND)
    assert got.status == (vfb_b200.OK if want["status"] == oracle.FOUND else vfb_b200.NOT_FOUND)
    assert got.size == want["size"]
    assert got.level_cands == want["level_cands"]
    if got.status == vfb_b200.OK:
        assert got.rpn == want["rpn"]
        assert got.solution_index == want["solution_index"]
    return got


@pytest.mark.parametrize("inst", cases.small_exact_cases(), ids=lambda i: i.name)
def test_exhaustive_equals_oracle(engine, inst):
    got = _check(engine, inst)
    # exact keys: the cached search returns the same first formula
    if got.status == vfb_b200.OK:
        cached = engine.solve(vfb_b200.Problem.from_instance(inst))
        assert cached.rpn == got.rpn


def test_exhaustive_not_found(engine):
    inst = cases.random_instance(4242, 2, 2, 2, 5, 5)
    inst.neg[0] = inst.pos[0]   # contradictory sample: nothing solves it
    got = _check(engine, inst)
    assert got.status == vfb_b200.NOT_FOUND


@pytest.mark.parametrize("run", [r for r in RUNS if r["max_size"] <= 10], ids=lambda r: r["name"])
def test_exhaustive_pins_reference_nocache(engine, run):
    # the reference returns a solution of the first solving size and operator
    # block; the first solution of the numbering has both
    inst = instance_from_json(run["json"], run["max_size"])
    ref_rpn = reference.parse_infix(run["nocache"]["formula"], inst.names)
    want = oracle.exhaustive(oracle.Problem.from_instance(inst), 1 << 26)
    if want["status"] != oracle.FOUND:
        pytest.skip("beyond the oracle's enumeration budget")
    got = engine.solve_exhaustive(vfb_b200.Problem.from_instance(inst))
    assert got.status == vfb_b200.OK
    assert got.size == len(ref_rpn)
    assert got.rpn[-1] == ref_rpn[-1]
    assert got.rpn == want["rpn"]


def test_cli_nocache(engine, tmp_path):
    inst = synth.config_small()
    path = tmp_path / "small.json"
    inst.write_json(str(path))
    cli = os.path.join(os.path.dirname(vfb_b200.LIB_PATH), "vfb")
    out = subprocess.run([cli, str(path), "10", "--nocache", "--quiet"], capture_output=True, text=True)
    assert out.returncode == 0
    got = engine.solve_exhaustive(vfb_b200.Problem.from_instance(synth.config_small()))
    assert out.stdout.strip() == f"{path}, {got.infix(inst.names)}"
