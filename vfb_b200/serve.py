"""Serving loop: continuous batching of arriving solve requests.

run_stream() replays a request stream -- (arrival time in seconds, Problem)
pairs -- against one engine in real time: a request is submitted once the wall
clock passes its arrival time, every vfb_serve_step admits queued requests
into free device slots (while the memory held stays under budget) and builds
one more level of every resident instance, and finished results come back
with their tags.  Requests that arrive while others are on the GPU join at the
next level boundary.  Latency = completion time - arrival time.

  python -m vfb_b200.serve --rate 100 --count 2000 [--slots 256]
  python -m vfb_b200.serve --rates 10,20,50,100,200,500 --window 20

Large-shape requests (8 APs, 63 traces of length 64) grow until their buffers
reach the per-request cap (--request-gb, default a quarter of the budget) and
then finish with status LIMIT and the sizes they completed; the output counts
them apart from the solved ones.
"""
from __future__ import annotations

import argparse
import json
import statistics
import time

from . import Engine, Problem, synth


def percentile(xs, q):
    xs = sorted(xs)
    if not xs:
        return None
    i = min(len(xs) - 1, max(0, int(round(q / 100.0 * (len(xs) - 1)))))
    return xs[i]


def run_stream(engine: Engine, stream, slots: int = 256, max_traces: int = 64, max_steps: int = 0):
    """Returns (results by index, latencies by index, makespan seconds).
    max_steps > 0: raise RuntimeError after that many serve steps."""
    engine.serve_open(slots, max_traces)
    n = len(stream)
    results, finish = [None] * n, [0.0] * n
    nxt, done, steps = 0, 0, 0
    t0 = time.perf_counter()
    try:
        while done < n:
            steps += 1
            if max_steps and steps > max_steps:
                raise RuntimeError(f"stream not served within {max_steps} steps ({done}/{n} done)")
            now = time.perf_counter() - t0
            while nxt < n and stream[nxt][0] <= now:
                engine.serve_submit(stream[nxt][1], nxt)
                nxt += 1
            out, active, queued = engine.serve_step()
            t = time.perf_counter() - t0
            for tag, res in out:
                results[tag] = res
                finish[tag] = t
                done += 1
            if active == 0 and queued == 0 and nxt < n:
                # idle until the next arrival
                wait = stream[nxt][0] - (time.perf_counter() - t0)
                if wait > 0:
                    time.sleep(min(wait, 0.001))
    finally:
        engine.serve_close()
    lat = [finish[i] - stream[i][0] for i in range(n)]
    return results, lat, time.perf_counter() - t0


def request_stream(seed: int = 4, count: int = 2000, rate: float = 100.0, large_frac: float = 0.05):
    """(arrival, Problem) pairs: 95% mixed-batch shapes, 5% the large shape."""
    return [(t, Problem.from_instance(inst))
            for t, inst in synth.config_serving(seed, count, rate, large_frac)]


def summarize(rate, res, lat, span, slots, large=None):
    """Status counts, latency percentiles and throughput of one served stream;
    with large (a flag per request), the percentiles of the large-shape and
    the other requests apart as well."""
    by = {}
    for r in res:
        name = "missing" if r is None else {0: "found", 1: "not_found", 2: "limit", 3: "oom"}.get(
            r.status, "error")
        by[name] = by.get(name, 0) + 1
    return {"rate_req_per_s": rate, "requests": len(res), "status": by,
            "p50_ms": 1e3 * percentile(lat, 50), "p95_ms": 1e3 * percentile(lat, 95),
            "p99_ms": 1e3 * percentile(lat, 99), "mean_ms": 1e3 * statistics.mean(lat),
            "solves_per_s": len(res) / span, "makespan_s": span, "slots": slots,
            **({} if large is None else _by_class(lat, large))}


def _by_class(lat, large):
    out = {}
    for name, want in (("mixed", False), ("large", True)):
        sub = [x for x, f in zip(lat, large) if f == want]
        if sub:
            out[name] = {"requests": len(sub), "p50_ms": 1e3 * percentile(sub, 50),
                         "p95_ms": 1e3 * percentile(sub, 95), "p99_ms": 1e3 * percentile(sub, 99)}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--rate", type=float, default=100.0)
    ap.add_argument("--rates", type=str, default="",
                    help="comma-separated sweep; each rate replays min(count, window*rate) requests")
    ap.add_argument("--window", type=float, default=20.0, help="seconds of arrivals per swept rate")
    ap.add_argument("--count", type=int, default=2000)
    ap.add_argument("--slots", type=int, default=256)
    ap.add_argument("--seed", type=int, default=4)
    ap.add_argument("--large-frac", type=float, default=0.05)
    ap.add_argument("--request-gb", type=float, default=0.0, help="per-request cap (0: budget / 4)")
    ap.add_argument("--step-cands", type=int, default=1 << 23,
                    help="operator candidates of one request per step (0: whole levels)")
    args = ap.parse_args()
    rates = [float(x) for x in args.rates.split(",")] if args.rates else [args.rate]
    eng = Engine()
    eng.serve_limits(0.8, int(args.request_gb * (1 << 30)), args.step_cands)
    for rate in rates:
        count = args.count if not args.rates else min(args.count, max(50, int(args.window * rate)))
        insts = synth.config_serving(args.seed, count, rate, args.large_frac)
        stream = [(t, Problem.from_instance(inst)) for t, inst in insts]
        large = [inst.name == "large" for _, inst in insts]
        # warm the kernels (module load, graph capture) outside the measured stream
        run_stream(eng, [(0.0, p) for _, p in stream[:4] if p.num_traces < 63] or stream[:1], args.slots)
        res, lat, span = run_stream(eng, stream, args.slots)
        print(json.dumps(summarize(rate, res, lat, span, args.slots, large)), flush=True)
    eng.close()


if __name__ == "__main__":
    main()
