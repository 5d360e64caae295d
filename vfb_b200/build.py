"""Builds the sm_100a engine library and the `vfb` command in-tree.

Outputs (git-ignored, shipped with the source tree):
  vfb_b200/_lib/libvfb_b200.so   CUDA kernels + host driver + C ABI (include/vfb.h)
  vfb_b200/_lib/vfb              the JSON command-line front end
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_lib")
OBJ = os.path.join(ROOT, "_build", "vfb_b200")
LIB = os.path.join(OUT, "libvfb_b200.so")
CLI = os.path.join(OUT, "vfb")

NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I", os.path.join(ROOT, "include")]

UNITS = ["vfb_kernels.cu", "vfb_engine.cu", "vfb_io.cpp", "vfb_noalloc.cu", "vfb_synth.cpp", "vfb_exhaustive.cu",
         "vfb_bs.cu"]
HEADERS = ["vfb_device.cuh", "vfb_kernels.cuh", "vfb_ops.cuh"]


def _newer(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {cmd[0]} {os.path.basename(cmd[-1])}")


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OUT, exist_ok=True)
    os.makedirs(OBJ, exist_ok=True)
    hdrs = [os.path.join(SRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "vfb.h")]
    jobs = []
    objs = []
    for u in UNITS:
        src = os.path.join(SRC, u)
        obj = os.path.join(OBJ, u + ".o")
        objs.append(obj)
        if force or _newer(obj, [src] + hdrs):
            jobs.append([NVCC, *ARCH, *FLAGS, "-c", src, "-o", obj])
    with ThreadPoolExecutor(max_workers=len(UNITS)) as ex:
        list(ex.map(_run, jobs))
    if force or _newer(LIB, objs):
        _run([NVCC, *ARCH, "-shared", "-o", LIB, *objs])
    cli_src = os.path.join(SRC, "vfb_cli.cpp")
    if force or _newer(CLI, [cli_src, LIB]):
        _run(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"), cli_src, "-o", CLI,
              "-L", OUT, "-lvfb_b200", "-Wl,-rpath,$ORIGIN"])
    if verbose:
        print(LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
