"""Benchmark: unique characteristic sets per second and time-to-formula of the
cached LTL search on the planted single-instance workload (4 propositions,
20 positive + 20 negative traces of length 16 labelled by a uniformly drawn
size-9 formula, max size 13, relaxed hash keys), one solve per step.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl vfb|reference]

value   unique CS per second of device time: each solve's span on the engine's
        stream (CUDA events from the first upload to the last result read).
e2e     the same metric through the public C ABI (vfb_solve with host buffers,
        uploads and result read-back inside), host wall clock per call.
roofline  the dominant kernel of a profiling pass over the same steps (CUDA
        events around every launch on the engine's stream), algorithmic bytes
        per launch over its mean duration, against the measured HBM copy peak.
candidates_per_s  operator candidates evaluated (the per-level candidate
        counts up to the solution, as the reference's CheckedLTLs) per second
        of device time.
cpu_baseline  the CPU restatement (single thread) on a bounded sample.
--impl reference  the CPU restatement with OpenMP on every host core, same
        workload and metric (the reference itself is CUDA-only).

--no-tune  keep the built-in k_p1 launch shape instead of autotuning it on
        each workload first (for launch-list captures: the tuner's own solves
        are many thousands of launches).

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
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

WORKLOAD = ("planted-9: 4 APs, 20+20 traces of length 16 (Bernoulli 0.5) labelled by a uniformly "
            "drawn size-9 formula (seed 1), max size 13, relaxed 128-bit hash keys")
METRIC = "unique characteristic sets per second (cached bottom-up LTL search, time-to-formula)"
UNIT = "unique CS/s"


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:  # noqa: BLE001
        return 6650.0, "fallback"


def _traffic(kernel: str):
    try:
        with open(os.path.join(ROOT, "profiles", "roofline_traffic.json")) as f:
            return json.load(f).get(kernel)
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


def run_reference(args, inst):
    """CPU restatement with OpenMP on every host core (rank 0 only)."""
    import oracle
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
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
        "data": "synthetic", "config": {"workload": WORKLOAD, "l2": "n/a (host run)"},
        "time_to_formula_ms": 1e3 * statistics.median(times),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"{args.steps} full solves of the workload (OpenMP, {cores} threads)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


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
    p = vfb_b200.Problem.from_instance(synth.config_batch(count=3)[2])
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
    return {"instance": "mixed batch #2 (7 APs, 36 traces, size 9, 11.3M unique CS)",
            "kernel": name, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "ms": ms, "launches": nl, "unique_cs": r.total_rows,
            "kernels": per, "autotuned": tuned}


def cpu_baseline(inst, budget_s: float):
    import oracle
    prob = oracle.Problem.from_instance(inst, threads=1)
    units, t_total, n = 0, 0.0, 0
    while t_total < budget_s or n == 0:
        t0 = time.perf_counter()
        r = oracle.solve(prob)
        t_total += time.perf_counter() - t0
        units += r["total_rows"]
        n += 1
    return {"value": units / t_total, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"{n} full solves of the workload, single thread ({t_total:.1f} s)"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="vfb", choices=["vfb", "reference"])
    ap.add_argument("--cpu-budget", type=float, default=10.0)
    ap.add_argument("--no-tune", action="store_true")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    world, rank, local = _dist()

    from vfb_b200 import synth
    inst = synth.config_planted()

    if args.impl == "reference":
        if rank == 0:
            run_reference(args, inst)
        return

    import torch
    if world > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", init_method="env://",
                                timeout=__import__("datetime").timedelta(seconds=120))
    else:
        torch.cuda.set_device(local)
    import vfb_b200
    prob = vfb_b200.Problem.from_instance(inst)
    eng = vfb_b200.Engine(device=local)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")   # > 126 MB L2
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
    eng.close()

    # profiling pass: per-kernel CUDA-event times over the same solves
    peng = vfb_b200.Engine(device=local, profile=True)
    peng.set_tune(table)   # None: built-in
    for _ in range(args.warmup):
        peng.solve(prob)
    peng.profile_reset()
    for _ in range(args.steps):
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
    dom = max(prof, key=lambda p: p[2]) if prof else None
    roof = None
    if dom:
        name, nl, ms, nbytes = dom
        per_launch_s = ms * 1e-3 / nl
        achieved = (nbytes / nl) / per_launch_s / 1e9 if per_launch_s > 0 else 0.0
        roof = {"kernel": name, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_kind": peak_kind,
                "traffic": _traffic(name), "bytes_per_launch": nbytes / nl,
                "us_per_launch": per_launch_s * 1e6, "launches": nl,
                "share_of_kernel_time": ms / sum(p[2] for p in prof)}

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
        "candidates_per_s": world * cands / dev_total,
        "time_to_formula_device_ms": 1e3 * statistics.median(dev_s),
        "formula": answer,
        "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": h2d // args.steps,
                "d2h_bytes_per_step": d2h // args.steps},
        "gpu_launches": launches,
        "roofline": roof,
        "kernels": [{"name": p[0], "launches": p[1], "ms": p[2], "bytes": p[3]} for p in prof],
        "clocks": clk.summary(),
    }
    line["batched"] = batched(local, flush, tune=not args.no_tune)
    line["large_instance"] = large_roofline(local, peak, tune=not args.no_tune)
    line["cpu_baseline"] = cpu_baseline(inst, args.cpu_budget)
    print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
