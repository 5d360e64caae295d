"""Command line: write a synthetic workload instance as trace JSON.

  python -m vfb_b200 synth small|planted|large|batch [--index I] [--seed S] --out FILE

The file has the reference's trace schema (ExampleLTLF.json), so it can be
solved with the drop-in CLI (`vfb_b200/_lib/vfb FILE N`) or the reference's
own programs; the workload's max size N is printed on stderr.  `batch --index I` is instance I of the mixed
batch (seed 3 unless --seed is given).
"""
from __future__ import annotations

import argparse
import sys

from . import synth


def main(argv=None):
    ap = argparse.ArgumentParser(prog="python -m vfb_b200")
    sub = ap.add_subparsers(dest="cmd", required=True)
    sp = sub.add_parser("synth", help="write one synthetic instance as trace JSON")
    sp.add_argument("config", choices=["small", "planted", "large", "batch"])
    sp.add_argument("--index", type=int, default=0)
    sp.add_argument("--seed", type=int, default=None)
    sp.add_argument("--out", required=True)
    args = ap.parse_args(argv)
    if args.config == "small":
        inst = synth.config_small(0 if args.seed is None else args.seed)
    elif args.config == "planted":
        inst = synth.config_planted(1 if args.seed is None else args.seed)
    elif args.config == "large":
        inst = synth.config_large(2 if args.seed is None else args.seed)
    else:
        inst = synth.config_batch(3 if args.seed is None else args.seed, count=args.index + 1)[args.index]
    inst.write_json(args.out)
    print(f"{args.out}: {inst.num_vars} APs, {len(inst.pos)}+{len(inst.neg)} traces, "
          f"max size {inst.max_size}", file=sys.stderr)


if __name__ == "__main__":
    main()
