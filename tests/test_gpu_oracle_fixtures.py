"""GPU parity on the benchmark workloads against the oracle's committed results
(tests/golden/oracle_batch.json, written by tests/golden/make_oracle_fixtures.py).

* the mixed batch (256 instances, seed 3): vfb_batch_solve and one vfb_solve
  per instance, both bit-exact with the oracle's restatement of LTLI
  (LTL_BS.cu:1069-1532) in the canonical order;
* the large shape (8 APs, 31+32 traces of length 64): seed 2 (solved by one
  proposition) and seed 7 to size 17, the deep seed to the oracle's size 9;
  the deep seed's full search under the 150 GB budget: its stored levels equal
  the oracle's, its formula is a solution (the oracle's evaluator), and its
  size is above 9, the oracle's proof that nothing smaller exists;
* the memory budget: with a budget (5 GB) that holds levels 1-8 of the deep seed but
  not level 9, level 9 is tested without being stored (LTL_BS's onTheFly,
  LTL_BS.cu:331-349) and the search ends with VFB_LIMIT after it;
* the head of the serving stream (seed 4): 64 requests served together by the
  continuous-batching loop, each equal to the oracle's result.
"""
import json
import os

import pytest

import oracle
import vfb_b200
from vfb_b200 import serve, synth

pytestmark = pytest.mark.gpu

FIX = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "oracle_batch.json")


@pytest.fixture(scope="module")
def fixture():
    with open(FIX) as f:
        return json.load(f)


def _key(r):
    if isinstance(r, dict):
        return (r["status"], r["size"], r["rpn"], r["level_rows"], r["level_cands"], r["solution_index"],
                r["total_rows"])
    return (r.status, r.size, r.rpn, r.level_rows, r.level_cands, r.solution_index, r.total_rows)


@pytest.fixture(scope="module")
def batch_probs():
    return [vfb_b200.Problem.from_instance(i) for i in synth.config_batch()]


def test_mixed_batch_matches_oracle(engine, fixture, batch_probs):
    got = engine.batch_solve(batch_probs)
    want = fixture["batch"]
    assert len(got) == len(want) == 256
    bad = [w["name"] for g, w in zip(got, want) if _key(g) != _key(w)]
    assert not bad, bad


def test_mixed_batch_solo_matches_oracle(engine, fixture, batch_probs):
    bad = [w["name"] for p, w in zip(batch_probs, fixture["batch"]) if _key(engine.solve(p)) != _key(w)]
    assert not bad, bad


def _large_engine():
    return vfb_b200.Engine(mem_limit_bytes=synth.LARGE_MEM_BYTES)


def test_large_shape_matches_oracle(fixture):
    want = {r["name"]: r for r in fixture["large"]}
    deep = f"large-s{synth.LARGE_DEEP_SEED}"
    with _large_engine() as eng:
        for name, inst in (("large-s2", synth.config_large(2)), ("large-s7", synth.config_large(7)),
                           (deep, synth.config_large_deep(max_size=fixture["large_oracle_max"]))):
            got = eng.solve(vfb_b200.Problem.from_instance(inst))
            assert _key(got) == _key(want[name]), name


def test_large_deep_full_search(fixture):
    """The headline workload's search: levels 1-9 as the oracle stores them,
    then a formula that the oracle's evaluator accepts, larger than 9."""
    want = {r["name"]: r for r in fixture["large"]}[f"large-s{synth.LARGE_DEEP_SEED}"]
    top = fixture["large_oracle_max"]
    assert want["status"] == oracle.NOT_FOUND and want["size"] == top
    inst = synth.config_large_deep()
    with _large_engine() as eng:
        got = eng.solve(vfb_b200.Problem.from_instance(inst))
        again = eng.solve(vfb_b200.Problem.from_instance(inst))
    assert got.status == vfb_b200.OK
    assert got.size > top
    assert got.level_rows[:top] == want["level_rows"]
    assert got.level_cands[:top] == want["level_cands"]
    ok, _ = oracle.eval_rpn(oracle.Problem.from_instance(inst), got.rpn)
    assert ok == 1
    assert len(got.rpn) == got.size
    assert _key(again) == _key(got)


def test_budget_switches_to_on_the_fly(fixture):
    """Levels 1-8 of the deep seed take about 2 GB; a 5 GB budget cannot hold
    level 9 (24 M more rows of 64 words), so level 9's 44.5 M candidates are
    tested without being stored, hold no solution, and the search ends there
    with the eight stored sizes."""
    want = {r["name"]: r for r in fixture["large"]}[f"large-s{synth.LARGE_DEEP_SEED}"]
    inst = synth.config_large_deep()
    with vfb_b200.Engine(mem_limit_bytes=5 << 30) as eng:
        got = eng.solve(vfb_b200.Problem.from_instance(inst))
    assert got.status == vfb_b200.LIMIT
    # the sizes reported are the stored ones (LIMIT: the on-the-fly level held nothing)
    assert got.size == 8
    assert got.level_rows == want["level_rows"][:8]
    assert got.level_cands == want["level_cands"][:8]


def test_serving_head_matches_oracle(engine, fixture):
    head = fixture["serving"]
    insts = [inst for _, inst in synth.config_serving(count=fixture["serve_head"])]
    stream = []
    for inst, rec in zip(insts, head):
        inst.max_size = rec["max_size"]          # large-shape requests: the fixture's limit
        stream.append((0.0005 * len(stream), vfb_b200.Problem.from_instance(inst)))
    results, lat, _ = serve.run_stream(engine, stream, slots=32)
    bad = [rec["name"] for got, rec in zip(results, head) if got is None or _key(got) != _key(rec)]
    assert not bad, bad
    assert all(x >= 0 for x in lat)
