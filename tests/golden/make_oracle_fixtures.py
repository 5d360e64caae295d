"""Writes the oracle's results for the mixed batch and for the head of the
serving stream to tests/golden/oracle_batch.json (CPU only, a few minutes on
8 cores).

  mixed batch   all 256 instances of the batched workload (seed 3): APs 2-8,
                traces 4-63, lengths 4-64 per trace, planted size 5-11,
                max size planted+4
  large shape   the large single instance (8 APs, 31+32 traces of length 64,
                planted size 13) at seed 2 (to size 17), at seed 7 (to size 17)
                and at the deep seed (synth.LARGE_DEEP_SEED) to size
                LARGE_ORACLE_MAX, the largest size the oracle finishes here in
                well under a minute (24 M characteristic sets)
  serving head  the first SERVE_HEAD requests of the serving stream (seed 4):
                95% drawn like the mixed batch, 5% in the large shape (8 APs,
                31+32 traces of length 64); the large-shape requests are
                searched to size SERVE_LARGE_MAX only, so that the oracle
                finishes them (the GPU tests submit them with the same limit)

Each record holds what the GPU path must reproduce bit for bit: status, size,
RPN, unique characteristic sets and candidates per size, the solution's
canonical index and the total.  The oracle restates LTLI (LTL_BS.cu:1069-1532)
in the canonical order; the GPU tests compare vfb_batch_solve, vfb_solve and
the serving loop with these records.

Usage:  python tests/golden/make_oracle_fixtures.py
"""
from __future__ import annotations

import json
import os
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from vfb_b200 import synth  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "oracle_batch.json")
SERVE_HEAD = 64
SERVE_LARGE_MAX = 8
LARGE_ORACLE_MAX = 9


def serve_head():
    """(name, instance) of the first SERVE_HEAD serving requests, large-shape
    ones limited to SERVE_LARGE_MAX."""
    out = []
    for i, (_, inst) in enumerate(synth.config_serving(count=SERVE_HEAD)):
        if inst.num_vars == 8 and inst.num_traces == 63 and set(inst.lengths()) == {64}:
            inst.max_size = min(inst.max_size, SERVE_LARGE_MAX)
        out.append((f"serve{i}", inst))
    return out


def record(name, inst, threads):
    r = oracle.solve(oracle.Problem.from_instance(inst, threads=threads))
    return {"name": name, "max_size": inst.max_size, "status": r["status"], "size": r["size"],
            "rpn": r["rpn"], "level_rows": r["level_rows"], "level_cands": r["level_cands"],
            "solution_index": r["solution_index"], "total_rows": r["total_rows"]}


def main():
    threads = os.cpu_count() or 1
    t0 = time.time()
    batch = [record(i.name, i, threads) for i in synth.config_batch()]
    print(f"batch: {len(batch)} instances, {sum(r['total_rows'] for r in batch)} unique CS, "
          f"{time.time() - t0:.0f} s", flush=True)
    t0 = time.time()
    large = [record("large-s2", synth.config_large(2), threads),
             record("large-s7", synth.config_large(7), threads),
             record(f"large-s{synth.LARGE_DEEP_SEED}", synth.config_large_deep(max_size=LARGE_ORACLE_MAX),
                    threads)]
    print(f"large shape: {[(r['name'], r['status'], r['size']) for r in large]}, {time.time() - t0:.0f} s",
          flush=True)
    t0 = time.time()
    serve = [record(n, i, threads) for n, i in serve_head()]
    print(f"serving head: {len(serve)} requests, {time.time() - t0:.0f} s", flush=True)
    with open(OUT, "w") as f:
        json.dump({"generated_by": "tests/golden/make_oracle_fixtures.py",
                   "serve_head": SERVE_HEAD, "serve_large_max": SERVE_LARGE_MAX,
                   "large_oracle_max": LARGE_ORACLE_MAX, "deep_seed": synth.LARGE_DEEP_SEED,
                   "batch": batch, "large": large, "serving": serve}, f, separators=(",", ":"))
        f.write("\n")
    print("wrote", OUT)


if __name__ == "__main__":
    main()
