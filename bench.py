"""Benchmark: unique characteristic sets per second and time-to-formula of the
cached LTL search on the large planted instance (8 propositions, 31 positive
+ 32 negative traces of length 64, bits Bernoulli(0.3), labelled by a
uniformly drawn size-13 formula; max size 17; level cache plus hash set
capped at 150 GB of device memory, a level that does not fit being tested
without being stored), one solve per step.

The large shape at seed 2 is solved by one proposition (a 1-level search of 8
characteristic sets), so the headline runs the same shape at seed 12, the
first seed from 2 whose instance has no formula of size 9 or less
(vfb_b200.synth.LARGE_DEEP_SEED): 28 M characteristic sets stored over sizes
1-9, then size 10 searched up to its solution (129 M candidates, 83.9 M new
sets); its projected rows do not fit the 150 GB budget, so the level runs
without them and its solution is settled before any row is written.  The
seed-2 solve is reported under "large_seed2".

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl vfb|reference]

value   unique CS per second of device time: each solve's span on the engine's
        stream (CUDA events from the first upload to the last result read);
        the L2 is flushed before every solve (256 MB write).
e2e     the same metric through the public C ABI (vfb_solve with host
        buffers, uploads and result read-back inside), host wall clock.
roofline  the dominant kernel of a profiling pass over the same solves (CUDA
        events around every launch on the engine's stream): algorithmic bytes
        per launch by the per-candidate byte model of the scope table (operand
        rows, key probe, stored rows of the level's unique fraction) over its
        mean duration, against the measured HBM copy peak; "models" gives the
        same kernel under the engine's own byte count and its issue-rate bound
        (warp instructions per candidate from the committed ncu capture, over
        the SM issue peak at the sampled clock).
cpu_baseline  the CPU restatement (single thread) on a bounded sample: the
        same instance searched to size 8.
--impl reference  the CPU restatement with OpenMP on every host core, same
        instance and metric, each step the search to size 8 (the full search
        holds 28 M sets and a 129 M-candidate pass; the reference's own
        programs are CUDA-only and reject traces of length 64, LTL_BS.cu:1105).

Extra keys of the line: "large_seed2" (the shape's own seed), "batched" (the
256-instance mixed batch against 256 serial solves), "large_instance" (per-
kernel profile of the mixed batch's largest instance), "serving" (the Poisson
request stream, 2000 requests per rate, p50/p95/p99, engine budget 64 GiB;
500 req/s is replayed twice so that the line shows how much its tail moves
between runs), "reference_cuda" (the
reference's LTL_BS built for this GPU, timed on the planted 20+20 instance
where its recorded runs completed).

--no-tune   keep the built-in k_p1 launch shape (launch-list captures).
--quick     headline only (no extra keys).

N > 1 (torchrun): replicas -- every rank solves its own copy on its GPU; value
is the units of all ranks over the slowest rank's time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

WORKLOAD = ("large planted instance, deep seed: 8 APs, 31+32 traces of length 64 (Bernoulli 0.3) labelled by "
            "a uniformly drawn size-13 formula, seed 12 (the first seed from 2 with no formula of size <= 9; "
            "seed 2 is solved by one proposition), max size 17, level cache + hash set capped at 150 GB "
            "(a level that does not fit is tested without being stored), relaxed 128-bit hash keys")
METRIC = "unique characteristic sets per second (cached bottom-up LTL search, time-to-formula)"
UNIT = "unique CS/s"
SAMPLE_SIZE = 8      # CPU legs: the instance searched to this size
SERVE_RATES = "500,500,200,100,50"   # 500 req/s twice: the tails' run-to-run spread
SERVE_MEM_BYTES = 64 << 30          # serving engine budget (a quarter of it per request)


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:  # noqa: BLE001
        return 6650.0, "fallback"


def _profile_json(name: str):
    try:
        with open(os.path.join(ROOT, "profiles", name)) as f:
            return json.load(f)
    except Exception:  # noqa: BLE001
        return None


class ClockSampler:
    """nvidia-smi sampling during the timed region (SM clock, reasons)."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:  # noqa: BLE001
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:  # noqa: BLE001
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                mx = max(mx, float(parts[1]))
            except ValueError:
                continue
            for n, v in zip(names, parts[4:8]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def _dist():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def _allreduce_max(x: float, world: int) -> float:
    """Maximum over the ranks (the slowest replica's time)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(units_per_rank: int, seconds_per_rank: float, world: int) -> float:
    """Whole-job throughput of N replicas: the units of all ranks (each rank
    solves the same workload) over the slowest rank's time."""
    slowest = _allreduce_max(seconds_per_rank, world)
    return world * units_per_rank / slowest


def _barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


# ----------------------------------------------------------------- byte models
def level_blocks(level_rows, k: int, cands: int):
    """Candidates of level k by operator kind in the canonical order (blocks
    ~ & | X F G U; & and | over left sizes 1..(k-1)/2, U over every split),
    truncated to the first `cands` (a level that ends at its solution).
    Returns (unary, and_or, until)."""
    n = [0] + list(level_rows)          # n[i]: unique rows of size i
    un = n[k - 1]
    com = sum(n[i] * n[k - 1 - i] for i in range(1, (k - 1) // 2 + 1))
    ncom = sum(n[i] * n[k - 1 - i] for i in range(1, k - 1))
    counts = {"u": 0, "b": 0, "U": 0}
    left = cands
    for kind, size in (("u", un), ("b", com), ("b", com), ("u", un), ("u", un), ("u", un), ("U", ncom)):
        take = min(left, size)
        counts[kind] += take
        left -= take
    return counts["u"], counts["b"], counts["U"]


def scope_bytes(num_traces: int, level_rows, level_cands, tile_rows: int = 16):
    """Algorithmic bytes of each level by the per-candidate model of the scope
    table: unary 8T + 16 + u(8T+24); & | 8T + 8T/TILE_L + 16 + u(8T+24); U per
    pair 8T + 8T/TILE_L, per orientation 16 + u(8T+24), with u the level's
    unique fraction.  A level tested without being stored (rows 0) moves only
    its operands (no key probe, no row written).  Returns {level: bytes}."""
    T8 = 8.0 * num_traces
    out = {}
    for k in range(2, len(level_cands) + 1):
        c = level_cands[k - 1]
        if c == 0:
            continue
        rows = level_rows[k - 1]
        otf = rows == 0
        u = 0.0 if otf else rows / c
        per_unique = 0.0 if otf else 16.0 + u * (T8 + 24.0)
        nu, nb, nU = level_blocks(level_rows, k, c)
        out[k] = (nu * (T8 + per_unique) + nb * (T8 + T8 / tile_rows + per_unique)
                  + nU * ((T8 + T8 / tile_rows) / 2 + per_unique))
    return out


# ----------------------------------------------------------------- reference arm
def run_reference(args, world):
    """CPU restatement with OpenMP on every host core (rank 0 only): each step
    the deep instance searched to SAMPLE_SIZE.  The instance is drawn with the
    pure-Python generator, so this arm maps none of the engine's code."""
    import oracle
    from vfb_b200 import synth
    inst = synth.config_large_deep(max_size=SAMPLE_SIZE, native=False)
    cores = os.cpu_count() or 1
    prob = oracle.Problem.from_instance(inst, threads=cores)
    for _ in range(args.warmup):
        oracle.solve(prob)
    times, units = [], 0
    for _ in range(args.steps):
        t0 = time.perf_counter()
        r = oracle.solve(prob)
        times.append(time.perf_counter() - t0)
        units += r["total_rows"]
    tot = sum(times)
    value = units / tot
    sample = (f"each step: the workload's instance searched to size {SAMPLE_SIZE} "
              f"({units // args.steps} unique CS; the full search stores 28 M and tests 129 M more "
              f"candidates), OpenMP on {cores} threads")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
        "data": "synthetic", "config": {"workload": WORKLOAD, "l2": "n/a (host run)"},
        "time_to_formula_ms": 1e3 * statistics.median(times),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------- extra legs
def _tune(eng, probs, sample: str, enabled: bool):
    """Autotune eng's launch shape on probs (when enabled); the summary for the line."""
    if not enabled:
        return {"sample": None, "bands": "built-in shape (--no-tune)"}
    return _tune_summary(eng.autotune(probs, reps=2), sample)


def _tune_summary(table: dict, sample: str) -> dict:
    """The autotuned k_p1 shape of the bands the sample's levels fell in:
    band -> [staged rows, log2 tile target, CTAs] (0: built-in), and the
    sample's k_p1 time under it against the built-in shape."""
    bands = {b: [table["rows"][b], table["tiles_log2"][b], table["blocks"][b]]
             for b in range(len(table["levels"])) if table["levels"][b]}
    return {"sample": sample, "bands": bands,
            "p1_ms_tuned": round(sum(table["ms"]), 4), "p1_ms_builtin": round(sum(table["ms_default"]), 4)}


def _tile_rows(table, cands: int) -> int:
    """Staged rows per k_p1 tile of a level of `cands` candidates under table."""
    b = 0
    while b < 15 and (cands >> (2 * b + 2)) != 0:
        b += 1
    r = table["rows"][b] if table else 0
    return min(r, 32) if r else 16


def large_seed2(local: int, flush, reps: int = 50):
    """The large shape at its own seed 2: one proposition separates the traces."""
    import torch
    import vfb_b200
    from vfb_b200 import synth
    inst = synth.config_large(2)
    p = vfb_b200.Problem.from_instance(inst)
    eng = vfb_b200.Engine(device=local, mem_limit_bytes=synth.LARGE_MEM_BYTES)
    for _ in range(3):
        eng.solve(p)
    dev, wall = [], []
    for _ in range(reps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = eng.solve(p)
        wall.append(time.perf_counter() - t0)
        dev.append(r.device_seconds)
    eng.close()
    return {"workload": "large planted instance at seed 2 (8 APs, 31+32 traces of length 64, max size 17)",
            "status": vfb_b200.STATUS_NAMES[r.status], "size": r.size, "formula": r.infix(inst.names),
            "unique_cs": r.total_rows, "time_to_formula_device_ms": 1e3 * statistics.median(dev),
            "time_to_formula_ms": 1e3 * statistics.median(wall), "reps": reps}


def batched(local: int, flush, count: int = 256, reps: int = 3, tune: bool = True):
    """The mixed batch (seed 3): one vfb_batch_solve of every instance against
    one vfb_solve per instance on the same engine, both warm (device timeline
    of every call summed over the run, torch synchronised around it)."""
    import torch
    import vfb_b200
    from vfb_b200 import synth
    probs = [vfb_b200.Problem.from_instance(i) for i in synth.config_batch(count=count)]
    eng = vfb_b200.Engine(device=local)
    tuned = _tune(eng, probs[:16], "the batch's first 16 instances, solved one by one", tune)
    key = lambda r: (r.status, r.size, r.rpn, r.level_rows, r.level_cands)  # noqa: E731
    serial = [eng.solve(p) for p in probs]        # warm-up (grows every buffer once)
    eng.batch_solve(probs)
    flush.zero_()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    serial = [eng.solve(p) for p in probs]
    ts = time.perf_counter() - t0
    tb = []
    same = True
    for _ in range(reps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        out = eng.batch_solve(probs)
        tb.append(time.perf_counter() - t0)
        same = same and all(key(a) == key(b) for a, b in zip(serial, out))
    eng.close()
    best = statistics.median(tb)
    return {"workload": f"mixed batch: {count} planted instances (seed 3), APs 2-8, traces 4-63, "
                        "lengths 4-64 per trace, planted size 5-11, max size planted+4",
            "solves_per_s": count / best, "ms_per_batch": 1e3 * best,
            "serial_solves_per_s": count / ts, "serial_ms": 1e3 * ts,
            "speedup_vs_serial": ts / best, "identical_to_serial": same,
            "unique_cs": sum(r.total_rows for r in serial), "reps": reps, "autotuned": tuned}


def large_roofline(local: int, peak: float, tune: bool = True):
    """Per-kernel profile of the largest instance of the mixed batch (#2,
    11.3M unique CS): the kernels' rates on levels that fill the GPU."""
    import vfb_b200
    from vfb_b200 import synth
    inst = synth.config_batch(count=3)[2]
    p = vfb_b200.Problem.from_instance(inst)
    eng = vfb_b200.Engine(device=local, profile=True)
    tuned = _tune(eng, [p], "the instance", tune)
    eng.solve(p)
    eng.solve(p)
    eng.profile_reset()
    r = eng.solve(p)
    prof = eng.profile()
    eng.close()
    name, nl, ms, nbytes = max(prof, key=lambda q: q[2])
    achieved = nbytes / (ms * 1e-3) / 1e9
    per = {}
    for q in prof:
        rate = q[3] / (q[2] * 1e-3) / 1e9 if q[2] > 0 and q[3] > 0 else None
        per[q[0]] = {"ms": round(q[2], 3), "launches": q[1],
                     "algorithmic_gbs": round(rate, 1) if rate else None,
                     "frac": round(rate / peak, 4) if rate else None}
    s8d = sum(scope_bytes(inst.num_traces, r.level_rows, r.level_cands).values())
    return {"instance": "mixed batch #2 (7 APs, 36 traces, size 9, 11.3M unique CS)",
            "kernel": name, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "ms": ms, "launches": nl, "unique_cs": r.total_rows,
            "scope_model_bytes": s8d,
            "scope_model_k_p1_gbs": s8d / (per["k_p1"]["ms"] * 1e-3) / 1e9 if "k_p1" in per else None,
            "kernels": per, "autotuned": tuned}


def serving(local: int, rates: str, count: int):
    """The serving stream (seed 4: 95% mixed-batch shapes, 5% the large shape)
    replayed in real time at each rate through the continuous-batching loop."""
    import vfb_b200
    from vfb_b200 import serve, synth
    eng = vfb_b200.Engine(device=local, mem_limit_bytes=SERVE_MEM_BYTES)
    eng.serve_limits(0.8, 0, 1 << 23)
    out = []
    for rate in [float(x) for x in rates.split(",") if x]:
        insts = synth.config_serving(4, count, rate, 0.05)
        stream = [(t, vfb_b200.Problem.from_instance(i)) for t, i in insts]
        large = [i.name == "large" for _, i in insts]
        serve.run_stream(eng, [(0.0, p) for _, p in stream[:4] if p.num_traces < 63] or stream[:1], 256)
        res, lat, span = serve.run_stream(eng, stream, 256)
        out.append(serve.summarize(rate, res, lat, span, 256, large))
    eng.close()
    return {"workload": f"Poisson request stream, seed 4, {count} requests per rate; 95% mixed-batch shapes, "
                        "5% the large shape (own seeds, max size 17); engine budget "
                        f"{SERVE_MEM_BYTES >> 30} GiB, per-request cap a quarter of it",
            "rates": out,
            "not_run": "rates 20 and 10 req/s (100 s and 200 s of arrivals): python bench.py --serve-rates 20,10"}


def reference_cuda(local: int, reps: int = 5):
    """The reference's LTL_BS built from its sources for sm_100a with its
    timing output, run on the planted 20+20 instance (4 APs, length 16, max
    size 13) with each relaxed rule: the inputs on which its recorded runs
    completed.  Its Running Time covers its LTLI call (allocation included).
    The same instance through this engine is timed beside it."""
    import vfb_b200
    from oracle import reference
    from vfb_b200 import synth
    if not reference.timed_available():
        return {"unavailable": "the reference's timed LTL_BS build (oracle/_ref/ltl_bs_timed) is missing"}
    inst = synth.config_planted()
    out = {"workload": "planted 20+20 instance (seed 1): 4 APs, traces of length 16, max size 13",
           "program": "LTL_BS.cu built with nvcc -arch=sm_100a -DMEASUREMENT_MODE; costs 1, "
                      "BS stage off, NegType 1", "runs": {}}
    env = dict(os.environ, CUDA_VISIBLE_DEVICES=str(local))
    with tempfile.TemporaryDirectory() as tmp:
        txt = os.path.join(tmp, "planted.txt")
        with open(txt, "w") as f:
            f.write(reference.instance_to_text(inst))
        for rlx in (1, 2, 3):
            secs, last = [], {}
            for _ in range(reps):
                last = reference.run_ltl_bs_timed(txt, 13, rlx, env=env)
                if last["returncode"] != 0 or last["seconds"] is None:
                    secs = []
                    break
                secs.append(last["seconds"])
            out["runs"][str(rlx)] = {"median_s": statistics.median(secs) if secs else None,
                                     "reps": len(secs), "returncode": last.get("returncode"),
                                     "cost": last.get("cost"), "formula": last.get("formula")}
    eng = vfb_b200.Engine(device=local)
    p = vfb_b200.Problem.from_instance(inst)
    for _ in range(3):
        eng.solve(p)
    dev, wall = [], []
    for _ in range(50):
        r = eng.solve(p)
        dev.append(r.device_seconds)
        wall.append(r.seconds)
    eng.close()
    out["this_engine"] = {"time_to_formula_device_ms": 1e3 * statistics.median(dev),
                          "time_to_formula_ms": 1e3 * statistics.median(wall), "size": r.size}
    return out


def cpu_baseline(budget_s: float):
    """Single-thread CPU restatement on the bounded sample (the deep
    instance searched to SAMPLE_SIZE), repeated for about budget_s."""
    import oracle
    from vfb_b200 import synth
    inst = synth.config_large_deep(max_size=SAMPLE_SIZE)
    prob = oracle.Problem.from_instance(inst, threads=1)
    units, t_total, n = 0, 0.0, 0
    while t_total < budget_s or n == 0:
        t0 = time.perf_counter()
        r = oracle.solve(prob)
        t_total += time.perf_counter() - t0
        units += r["total_rows"]
        n += 1
    return {"value": units / t_total, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"{n} searches of the workload's instance to size {SAMPLE_SIZE} "
                      f"({r['total_rows']} unique CS each), single thread ({t_total:.1f} s)"}


# ----------------------------------------------------------------- main
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="vfb", choices=["vfb", "reference"])
    ap.add_argument("--cpu-budget", type=float, default=10.0)
    ap.add_argument("--no-tune", action="store_true")
    ap.add_argument("--quick", action="store_true")
    ap.add_argument("--serve-rates", default=SERVE_RATES)
    ap.add_argument("--serve-count", type=int, default=2000)
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    world, rank, local = _dist()

    if args.impl == "reference":
        if rank == 0:
            run_reference(args, world)
        return

    import torch
    from vfb_b200 import synth
    if world > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", init_method="env://",
                                timeout=__import__("datetime").timedelta(seconds=120))
    else:
        torch.cuda.set_device(local)
    import vfb_b200
    inst = synth.config_large_deep()
    prob = vfb_b200.Problem.from_instance(inst)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")   # > 126 MB L2
    eng = vfb_b200.Engine(device=local, mem_limit_bytes=synth.LARGE_MEM_BYTES)
    # k_p1 launch shape per level band, tuned on the workload before timing
    table = eng.autotune([prob], reps=2) if not args.no_tune else None

    for _ in range(args.warmup):
        r = eng.solve(prob)
        assert r.status == vfb_b200.OK, r
    torch.cuda.synchronize()

    dev_s, wall_s, units, launches, h2d, d2h, cands = [], [], 0, 0, 0, 0, 0
    _barrier(world)
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            r = eng.solve(prob)
            wall_s.append(time.perf_counter() - t0)
            dev_s.append(r.device_seconds)
            units += r.total_rows
            cands += sum(r.level_cands)
            launches += r.kernel_launches
            h2d += r.h2d_bytes
            d2h += r.d2h_bytes
    torch.cuda.synchronize()
    _barrier(world)
    dev_total = _allreduce_max(sum(dev_s), world)
    wall_total = _allreduce_max(sum(wall_s), world)
    value = world * units / dev_total
    e2e = world * units / wall_total
    answer = r.infix(inst.names)
    final = r
    eng.close()

    # profiling pass: per-kernel CUDA-event times over the same solves
    psteps = min(args.steps, 5)
    peng = vfb_b200.Engine(device=local, profile=True, mem_limit_bytes=synth.LARGE_MEM_BYTES)
    peng.set_tune(table)   # None: built-in
    for _ in range(args.warmup):
        peng.solve(prob)
    peng.profile_reset()
    for _ in range(psteps):
        flush.zero_()
        torch.cuda.synchronize()
        peng.solve(prob)
    prof = peng.profile()
    peng.close()

    if rank != 0:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return

    peak, peak_kind = _peaks()
    clocks = clk.summary()
    roof = None
    kp1 = next((p for p in prof if p[0] == "k_p1"), None)
    dom = max(prof, key=lambda p: p[2]) if prof else None
    if dom:
        name, nl, ms, nbytes = dom
        per_launch_s = ms * 1e-3 / nl
        # the per-candidate byte model of the scope table, per solve, over the
        # levels k_p1 built (one launch per level)
        # (TILE_L: the staged rows of the largest level's band, which holds
        # most of the bytes)
        lvl_bytes = scope_bytes(inst.num_traces, final.level_rows, final.level_cands,
                                tile_rows=_tile_rows(table, max(final.level_cands)))
        s8d_per_solve = sum(lvl_bytes.values())
        s8d_per_launch = s8d_per_solve * psteps / nl if name == "k_p1" else None
        model = {"engine_bytes_per_launch": nbytes / nl,
                 "engine_gbs": (nbytes / nl) / per_launch_s / 1e9}
        if s8d_per_launch is not None:
            achieved = s8d_per_launch / per_launch_s / 1e9
            bytes_pl = s8d_per_launch
            basis = "scope-table per-candidate model (operand rows, key probe, unique fraction of stored rows)"
        else:
            achieved = model["engine_gbs"]
            bytes_pl = nbytes / nl
            basis = "engine byte count"
        traffic = _profile_json("roofline_traffic.json") or {}
        issue = _profile_json("k_p1_issue.json")
        if issue and kp1 and clocks.get("sm_mhz"):
            sms = issue.get("sms", 148)
            cand_per_solve = sum(final.level_cands[1:])
            inst_per_s = issue["warp_inst_per_candidate"] * cand_per_solve * psteps / (kp1[2] * 1e-3)
            peak_issue = sms * 4 * clocks["sm_mhz"] * 1e6
            model["issue"] = {"warp_inst_per_candidate": issue["warp_inst_per_candidate"],
                              "achieved_warp_inst_per_s": inst_per_s, "peak_warp_inst_per_s": peak_issue,
                              "frac": inst_per_s / peak_issue, "source": "profiles/k_p1_issue.json"}
        roof = {"kernel": name, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_kind": peak_kind, "basis": basis,
                "traffic": traffic.get(name), "bytes_per_launch": bytes_pl,
                "us_per_launch": per_launch_s * 1e6, "launches": nl,
                "share_of_kernel_time": ms / sum(p[2] for p in prof),
                "solve_gbs_scope_model": s8d_per_solve / statistics.median(dev_s) / 1e9,
                "models": model}

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * dev_total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
        "data": "synthetic",
        "config": {"workload": WORKLOAD, "parallelism": f"replicas{world}",
                   "l2": "flushed before every step (256 MB write)",
                   "launch_shape": _tune_summary(table, "the workload (autotuned before the warm-up)")
                   if table else {"sample": None, "bands": "built-in shape (--no-tune)"}},
        "time_to_formula_ms": 1e3 * statistics.median(wall_s),
        "time_to_formula_device_ms": 1e3 * statistics.median(dev_s),
        "candidates_per_s": world * cands / dev_total,
        "formula": answer, "size": final.size, "level_rows": final.level_rows,
        "level_cands": final.level_cands,
        "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": h2d // args.steps,
                "d2h_bytes_per_step": d2h // args.steps},
        "gpu_launches": launches,
        "roofline": roof,
        "kernels": [{"name": p[0], "launches": p[1], "ms": p[2], "bytes": p[3]} for p in prof],
        "clocks": clocks,
    }
    if not args.quick:
        line["large_seed2"] = large_seed2(local, flush)
        line["batched"] = batched(local, flush, tune=not args.no_tune)
        line["large_instance"] = large_roofline(local, peak, tune=not args.no_tune)
        del flush
        torch.cuda.empty_cache()
        line["serving"] = serving(local, args.serve_rates, args.serve_count)
        line["reference_cuda"] = reference_cuda(local)
    line["cpu_baseline"] = cpu_baseline(args.cpu_budget)
    print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
