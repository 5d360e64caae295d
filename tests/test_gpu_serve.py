"""Serving loop: requests admitted while others are on the GPU get exactly the
result a solo vfb_solve gives."""
import pytest

import vfb_b200
from vfb_b200 import serve, synth
from tests import cases

pytestmark = pytest.mark.gpu


def _key(r):
    return (r.status, r.size, r.rpn, r.level_rows, r.level_cands, r.solution_index)


def test_stream_results_equal_solo(engine):
    # a dense stream (all arrivals within a few ms) so requests overlap on the device
    stream = serve.request_stream(seed=11, count=40, rate=20000.0, large_frac=0.0)
    # one large-shape request of moderate size (8 APs, 63 traces of 64 steps, size 7)
    stream.insert(5, (stream[5][0], vfb_b200.Problem.from_instance(synth.config_large(13))))
    results, lat, span = serve.run_stream(engine, stream, slots=16)
    assert all(r is not None for r in results)
    for (t, prob), got in zip(stream, results):
        assert _key(got) == _key(engine.solve(prob))
    assert all(x >= 0 for x in lat)


def test_more_requests_than_slots(engine):
    insts = cases.planted_cases(6) + cases.small_exact_cases()[:6] + [synth.config_planted()]
    stream = [(0.0, vfb_b200.Problem.from_instance(i)) for i in insts]
    results, _, _ = serve.run_stream(engine, stream, slots=3)
    for (t, prob), got in zip(stream, results):
        assert _key(got) == _key(engine.solve(prob))


def test_growth_inside_a_stream(engine):
    inst = cases.random_instance(4242, 4, 5, 5, 16, 8)
    inst.neg[0] = inst.pos[0]
    big = vfb_b200.Problem.from_instance(inst)
    small = vfb_b200.Problem.from_instance(synth.config_small())
    stream = [(0.0, big), (0.0, small), (0.0, small)]
    results, _, _ = serve.run_stream(engine, stream, slots=2)
    assert _key(results[0]) == _key(engine.solve(big))
    assert results[1].status == vfb_b200.OK and results[2].status == vfb_b200.OK


def test_request_cap_ends_with_limit(engine):
    inst = cases.random_instance(4242, 4, 5, 5, 16, 8)
    inst.neg[0] = inst.pos[0]          # unsatisfiable: grows to max_size
    big = vfb_b200.Problem.from_instance(inst)
    small = vfb_b200.Problem.from_instance(synth.config_small())
    solo = engine.solve(big)
    try:
        engine.serve_limits(0.8, 1 << 20)
        results, _, _ = serve.run_stream(engine, [(0.0, big), (0.0, small)], slots=2)
    finally:
        engine.serve_limits(0.8, 0)
    got = results[0]
    assert got.status == vfb_b200.LIMIT
    assert 1 <= got.size < solo.size
    assert got.level_rows == solo.level_rows[:got.size]
    assert _key(results[1]) == _key(engine.solve(small))


def test_tight_budget_still_progresses(engine):
    # a budget every request exceeds: one request at a time, all complete
    insts = cases.planted_cases(4) + [synth.config_planted()]
    stream = [(0.0, vfb_b200.Problem.from_instance(i)) for i in insts]
    try:
        engine.serve_limits(1e-9, 0)
        results, _, _ = serve.run_stream(engine, stream, slots=4)
    finally:
        engine.serve_limits(0.8, 0)
    for (t, prob), got in zip(stream, results):
        assert _key(got) == _key(engine.solve(prob))


def test_sliced_levels_equal_solo(engine):
    # a tiny per-step slice: every level of every request takes many steps
    insts = [synth.config_planted(), cases.random_instance(4242, 4, 5, 5, 16, 8)] + cases.planted_cases(3)
    stream = [(0.0, vfb_b200.Problem.from_instance(i)) for i in insts]
    try:
        engine.serve_limits(0.8, 0, 2000)
        results, _, _ = serve.run_stream(engine, stream, slots=4)
    finally:
        engine.serve_limits(0.8, 0)
    for (t, prob), got in zip(stream, results):
        assert _key(got) == _key(engine.solve(prob))


def test_oversubscribed_memory_waits_instead_of_failing():
    # four requests admitted together whose buffers do not all fit the
    # budget at once: a growth that finds the memory held by the others waits
    # (or its request restarts later) instead of failing, so every result is
    # still the solo one
    probs = [vfb_b200.Problem.from_instance(i) for i in cases.unsatisfiable_cases()]
    with vfb_b200.Engine() as eng:
        full = [eng.solve(p) for p in probs]
    assert all(r.status == vfb_b200.NOT_FOUND for r in full)
    budget = cases.smallest_solo_budget(probs, full)   # holds each request alone
    assert budget is not None
    with vfb_b200.Engine(mem_limit_bytes=budget) as eng:
        # admit all four at once; no per-request cap below the device budget
        eng.serve_limits(1.0, 4 * budget)
        results, _, _ = serve.run_stream(eng, [(0.0, p) for p in probs], slots=4, max_steps=20000)
    for got, want in zip(results, full):
        assert _key(got) == _key(want)


@pytest.mark.parametrize("arena_mb", [2, 64])
def test_small_arena_falls_back_to_the_pool(engine, monkeypatch, arena_mb):
    # a serving session's buffers come from its arena, and from the pool when
    # no free range of the arena fits: with a tiny arena most growth takes the
    # pool path, blocks of both kinds are freed and reused within one session,
    # and every result is still the solo one
    monkeypatch.setenv("VFB_SERVE_ARENA_MB", str(arena_mb))
    insts = cases.planted_cases(5) + [synth.config_planted(), cases.random_instance(4242, 4, 5, 5, 16, 8)]
    insts += cases.small_exact_cases()[:5]
    stream = [(0.0005 * i, vfb_b200.Problem.from_instance(x)) for i, x in enumerate(insts)]
    results, _, _ = serve.run_stream(engine, stream, slots=4)
    for (t, prob), got in zip(stream, results):
        assert _key(got) == _key(engine.solve(prob))
