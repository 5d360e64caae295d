"""GPU parity: the CUDA engine (through the C ABI) against the CPU oracle.

Bit-exact: same status, minimal size, returned formula (RPN), per-size unique
counts, candidates evaluated and canonical solution index.
"""
import os
import subprocess

import pytest

import oracle
import vfb_b200
from vfb_b200 import synth
from tests import cases

pytestmark = pytest.mark.gpu


def _check(engine, inst, **kw):
    prob = vfb_b200.Problem.from_instance(inst)
    for k, v in kw.items():
        setattr(prob, k, v)
    got = engine.solve(prob)
    ref = oracle.solve(oracle.Problem.from_instance(inst, rlx_type=prob.rlx_type,
                                                    max_size=prob.max_size))
    status = {oracle.FOUND: vfb_b200.OK, oracle.NOT_FOUND: vfb_b200.NOT_FOUND}[ref["status"]]
    assert got.status == status
    assert got.size == ref["size"]
    assert got.rpn == ref["rpn"]
    assert got.level_rows == ref["level_rows"]
    assert got.level_cands == ref["level_cands"]
    if got.status == vfb_b200.OK:
        assert got.solution_index == ref["solution_index"]
        ok, _ = oracle.eval_rpn(oracle.Problem.from_instance(inst), got.rpn)
        assert ok == 1
    return got


def test_small_config(engine):
    _check(engine, synth.config_small())


@pytest.mark.parametrize("inst", cases.small_exact_cases(), ids=lambda i: i.name)
def test_exact_keys(engine, inst):
    _check(engine, inst)


@pytest.mark.parametrize("rlx", [1, 2, 3])
def test_relaxed_keys(engine, rlx):
    for inst in cases.relaxed_cases(rlx):
        _check(engine, inst, rlx_type=rlx)


@pytest.mark.parametrize("inst", cases.planted_cases(), ids=lambda i: i.name)
def test_planted(engine, inst):
    got = _check(engine, inst)
    assert got.size <= len(inst.planted)


def test_planted_config(engine):
    _check(engine, synth.config_planted())


def test_not_found_runs_every_level(engine):
    inst = cases.random_instance(77, 3, 3, 3, 6, 5)
    inst.neg[0] = inst.pos[0]          # a positive equal to a negative: unsolvable
    got = _check(engine, inst)
    assert got.status == vfb_b200.NOT_FOUND and got.size == 5


def test_length_64_traces(engine):
    inst = cases.random_instance(99, 2, 3, 3, 64, 5, p=0.3)
    _check(engine, inst)


def test_batch_equals_single(engine):
    insts = cases.planted_cases(5) + cases.small_exact_cases()[:5] + cases.relaxed_cases(3)[:2]
    probs = [vfb_b200.Problem.from_instance(i) for i in insts]
    batch = engine.batch_solve(probs)
    for p, b in zip(probs, batch):
        s = engine.solve(p)
        assert (b.status, b.size, b.rpn, b.level_rows, b.level_cands) == \
               (s.status, s.size, s.rpn, s.level_rows, s.level_cands)


def test_growth_path_large_level(engine):
    """An instance whose levels outgrow every initial buffer (rows, table,
    bitmap, tentative list) several times."""
    inst = cases.random_instance(4242, 4, 5, 5, 16, 9)
    inst.neg[0] = inst.pos[0]          # unsolvable: every level up to 9 is built
    got = _check(engine, inst)
    assert got.total_rows > 900_000


def test_cli_prints_reference_line(tmp_path):
    inst = synth.config_planted()
    path = tmp_path / "planted.json"
    inst.write_json(str(path))
    out = subprocess.run([vfb_b200.CLI_PATH, str(path), "13"], capture_output=True, text=True,
                         timeout=120)
    assert out.returncode == 0
    ref = oracle.solve(oracle.Problem.from_instance(inst))
    expect = synth.rpn_to_infix(ref["rpn"], inst.names)
    assert out.stdout == f"{path}, {expect}\n"


# ----------------------------------------------------------------- edge cases
def test_maximum_trace_count(engine):
    # 128 traces (the build's limit; the P1 tile holds 129-word rows)
    inst = cases.random_instance(7001, 3, 64, 64, [1 + (i * 7) % 12 for i in range(128)], 5)
    _check(engine, inst)


def test_maximum_proposition_count(engine):
    # 64 propositions: 64 level-1 rows, a size-5 solution
    inst = cases.random_instance(7137, 64, 10, 10, 8, 5)
    _check(engine, inst)


def test_duplicate_propositions(engine):
    inst = cases.random_instance(7003, 3, 3, 3, 8, 6)
    for _, words in inst.pos + inst.neg:
        words[2] = words[0]          # p2 is p0 on every trace
    _check(engine, inst)


def test_single_trace_and_one_sided_samples(engine):
    one = cases.random_instance(7004, 2, 1, 0, 5, 5)     # one positive trace only
    _check(engine, one)
    neg = cases.random_instance(7005, 2, 0, 3, 5, 5)     # negatives only
    _check(engine, neg)


def test_length_one_traces(engine):
    inst = cases.random_instance(7006, 3, 4, 4, 1, 6)
    _check(engine, inst)


def test_exact_key_boundary(engine):
    # trace lengths summing to exactly 126 bits (the last exact-key size) and
    # to 127 (the first relaxed one)
    _check(engine, cases.random_instance(7200, 2, 3, 3, [21] * 6, 7))
    _check(engine, cases.random_instance(7300, 2, 3, 3, [21] * 5 + [22], 7))


def test_on_the_fly_level(engine):
    # a memory budget that cannot hold the solution level's rows: its
    # candidates are tested without being stored, and the answer is the one
    # the unbounded search gives (LTL_BS's onTheFly mode)
    prob = vfb_b200.Problem.from_instance(synth.config_planted())
    full = engine.solve(prob)
    assert full.status == vfb_b200.OK
    hits = 0
    for mb in [4.0, 3.5, 3.0, 2.75, 2.5, 2.25, 2.0, 1.75, 1.5]:
        e = vfb_b200.Engine(mem_limit_bytes=int(mb * (1 << 20)))
        try:
            r = e.solve(prob)
        finally:
            e.close()
        if r.status == vfb_b200.OK and r.level_rows[-1] == 0:
            hits += 1
            assert (r.size, r.rpn, r.solution_index) == (full.size, full.rpn, full.solution_index)
            assert r.level_rows[:-1] == full.level_rows[:-1]
            assert r.level_cands == full.level_cands
        elif r.status == vfb_b200.OK:
            assert (r.size, r.rpn, r.level_rows) == (full.size, full.rpn, full.level_rows)
        elif r.status == vfb_b200.LIMIT:
            assert r.size < full.size and r.level_rows == full.level_rows[:r.size]
        else:
            assert r.status == vfb_b200.OOM
    assert hits >= 1


def test_second_context_gets_the_memory_the_first_released():
    # a context that solved many instances one by one keeps only its last
    # working set cached (not every superseded buffer size); a second context
    # created afterwards in the same process has the memory for the whole
    # batch and returns the same results
    probs = [vfb_b200.Problem.from_instance(i) for i in synth.config_batch(count=256)]
    key = lambda r: (r.status, r.size, r.rpn, r.level_rows, r.level_cands, r.solution_index)  # noqa: E731
    with vfb_b200.Engine() as first:
        want = [first.solve(p) for p in probs]
        with vfb_b200.Engine() as second:
            got = second.batch_solve(probs)
    assert [key(r) for r in got] == [key(r) for r in want]


def test_batch_under_memory_pressure_equals_solo():
    # eight instances in one batch under a budget that holds each alone but
    # not all of them: growths wait for memory, when every instance waits the
    # least advanced one starts again later, and (second call, with the final
    # sizes of the first as hints) instances whose first buffers do not fit
    # start when memory frees; every result is the solo one
    probs = [vfb_b200.Problem.from_instance(i)
             for i in cases.unsatisfiable_cases(seeds=range(4242, 4250))]
    with vfb_b200.Engine() as eng:
        full = [eng.solve(p) for p in probs]
    budget = cases.smallest_solo_budget(probs, full)
    assert budget is not None
    key = lambda r: (r.status, r.size, r.rpn, r.level_rows, r.level_cands)  # noqa: E731
    with vfb_b200.Engine(mem_limit_bytes=budget) as eng:
        got = eng.batch_solve(probs)
        again = eng.batch_solve(probs)      # with the capacity hints of the first call
    assert [key(r) for r in got] == [key(r) for r in full]
    assert [key(r) for r in again] == [key(r) for r in full]


@pytest.mark.parametrize("inst", cases.mirrored_cases() + cases.mirrored_cases(count=8, num_vars=8, length=20,
                                                                               max_size=7),
                         ids=lambda i: f"{i.name}_a{i.num_vars}")
def test_relaxed_key_collisions_on_the_solution(engine, inst):
    # the first solving candidate often shares its hash key with its earlier
    # mirror (which does not solve); candidates past it may have been skipped
    # by then, so the level is built again in full before the answer is read
    _check(engine, inst)


def test_relaxed_key_collisions_in_a_batch(engine):
    insts = cases.mirrored_cases(count=8, num_vars=8, length=20, max_size=7) + cases.mirrored_cases()
    probs = [vfb_b200.Problem.from_instance(i) for i in insts]
    key = lambda r: (r.status, r.size, r.rpn, r.level_rows, r.level_cands, r.solution_index)  # noqa: E731
    solo = [engine.solve(p) for p in probs]
    assert [key(r) for r in engine.batch_solve(probs)] == [key(r) for r in solo]


def test_relaxed_key_collisions_with_tiles_in_order():
    # one CTA takes the tiles in order, so every tile after the first
    # solution's skips the operators past it; where that solution turns out
    # not to own its key, the level is built again in full (this set has
    # several such levels) and the answer still equals the oracle's
    insts = cases.mirrored_cases() + cases.mirrored_cases(count=8, num_vars=8, length=20, max_size=7)
    insts += cases.mirrored_cases(count=24, num_vars=12, length=16, max_size=7)[8:]
    with vfb_b200.Engine() as eng:
        eng.set_tune({"rows": [1] * vfb_b200.TUNE_BANDS, "tiles_log2": [16] * vfb_b200.TUNE_BANDS,
                      "blocks": [1] * vfb_b200.TUNE_BANDS})
        for inst in insts:
            got = eng.solve(vfb_b200.Problem.from_instance(inst))
            ref = oracle.solve(oracle.Problem.from_instance(inst))
            assert got.rpn == ref["rpn"], inst.name
            assert got.level_rows == ref["level_rows"], inst.name
            assert got.level_cands == ref["level_cands"], inst.name
