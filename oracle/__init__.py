"""CPU oracle for VFB's cached LTL enumeration -- TEST INFRASTRUCTURE ONLY.

Imported by tests/, by the smoke check and by bench.py's CPU-baseline leg, and
nowhere else.  The product (vfb_b200) never imports it.

The C restatement lives in vfb_oracle.c; build() compiles it with gcc (OpenMP)
into oracle/_build/libvfb_oracle.so, and build_ref() compiles the reference's
own CUDA programs from their sources into oracle/_ref/ (used only to generate
golden fixtures on a GPU machine).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import time

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "libvfb_oracle.so")
OPS = "~&|XFGU"

MAX_SIZE = 32
FOUND, NOT_FOUND, LIMIT, BAD_INPUT = 0, 1, 2, 3
CANONICAL, REFCOMPAT = 0, 1


def build(force: bool = False) -> str:
    src = os.path.join(HERE, "vfb_oracle.c")
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(
            os.path.getmtime(src), os.path.getmtime(os.path.join(HERE, "vfb_oracle.h"))):
        subprocess.check_call(["gcc", "-O3", "-fopenmp", "-shared", "-fPIC", "-Wall",
                               "-o", LIB, src])
    return LIB


class _Problem(ctypes.Structure):
    _fields_ = [("num_traces", ctypes.c_int), ("num_pos", ctypes.c_int),
                ("num_vars", ctypes.c_int), ("max_size", ctypes.c_int),
                ("rlx_type", ctypes.c_int), ("mode", ctypes.c_int),
                ("threads", ctypes.c_int), ("ref_max_pitch", ctypes.c_int64),
                ("max_rows", ctypes.c_uint64),
                ("len", ctypes.POINTER(ctypes.c_uint8)),
                ("atoms", ctypes.POINTER(ctypes.c_uint64)),
                ("trace", ctypes.POINTER(ctypes.c_int64)), ("trace_cap", ctypes.c_int),
                ("cost", ctypes.c_int * 8), ("neg_type", ctypes.c_int)]


class _Result(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("size", ctypes.c_int),
                ("rpn_len", ctypes.c_int), ("rpn", ctypes.c_int16 * MAX_SIZE),
                ("level_rows", ctypes.c_uint64 * (MAX_SIZE + 1)),
                ("level_cands", ctypes.c_uint64 * (MAX_SIZE + 1)),
                ("solution_index", ctypes.c_uint64),
                ("total_rows", ctypes.c_uint64), ("seconds", ctypes.c_double),
                ("trace_len", ctypes.c_int)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = ctypes.CDLL(LIB)
        _lib.orc_solve.argtypes = [ctypes.POINTER(_Problem), ctypes.POINTER(_Result)]
        _lib.orc_exhaustive.argtypes = [ctypes.POINTER(_Problem), ctypes.c_uint64,
                                        ctypes.POINTER(_Result)]
        _lib.orc_eval_rpn.argtypes = [ctypes.POINTER(_Problem), ctypes.POINTER(ctypes.c_int16),
                                      ctypes.c_int, ctypes.POINTER(ctypes.c_uint64)]
        _lib.orc_make_key.argtypes = [ctypes.POINTER(_Problem), ctypes.POINTER(ctypes.c_uint64),
                                      ctypes.POINTER(ctypes.c_uint64),
                                      ctypes.POINTER(ctypes.c_uint64)]
        _lib.orc_apply.argtypes = [ctypes.POINTER(_Problem), ctypes.c_int,
                                   ctypes.POINTER(ctypes.c_uint64),
                                   ctypes.POINTER(ctypes.c_uint64),
                                   ctypes.POINTER(ctypes.c_uint64)]
        _lib.orc_ref_temp_capacity.argtypes = [ctypes.POINTER(_Problem)]
        _lib.orc_ref_temp_capacity.restype = ctypes.c_int64
    return _lib


class Problem:
    """Holds the ctypes arrays alive for one instance."""

    def __init__(self, lengths, atoms, num_pos, max_size, rlx_type=3,
                 mode=CANONICAL, threads=1, ref_max_pitch=2147483647,
                 max_rows=1 << 40, costs=None, neg_type=1):
        t = len(lengths)
        a = len(atoms)
        self._len = (ctypes.c_uint8 * t)(*lengths)
        flat = [w for row in atoms for w in row]
        self._atoms = (ctypes.c_uint64 * max(1, len(flat)))(*flat)
        self._trace = (ctypes.c_int64 * (5 * 4096))()
        self.p = _Problem(t, num_pos, a, max_size, rlx_type, mode, threads,
                          ref_max_pitch, max_rows,
                          ctypes.cast(self._len, ctypes.POINTER(ctypes.c_uint8)),
                          ctypes.cast(self._atoms, ctypes.POINTER(ctypes.c_uint64)),
                          ctypes.cast(self._trace, ctypes.POINTER(ctypes.c_int64)), 4096,
                          (ctypes.c_int * 8)(*(costs or [1] * 8)), neg_type)

    @classmethod
    def from_instance(cls, inst, **kw):
        kw.setdefault("rlx_type", inst.rlx_type)
        kw.setdefault("max_size", inst.max_size)
        return cls(inst.lengths(), inst.atom_words(), len(inst.pos), **kw)


def tokens(rpn_len, rpn):
    out = []
    for i in range(rpn_len):
        tk = rpn[i]
        out.append(tk if tk >= 0 else OPS[-tk - 1])
    return out


def _result(r: _Result) -> dict:
    k = r.size
    return {
        "status": r.status,
        "size": r.size,
        "rpn": tokens(r.rpn_len, r.rpn),
        "level_rows": [r.level_rows[i] for i in range(1, k + 1)],
        "level_cands": [r.level_cands[i] for i in range(1, k + 1)],
        "solution_index": r.solution_index,
        "total_rows": r.total_rows,
        "seconds": r.seconds,
    }


def solve(prob: Problem) -> dict:
    r = _Result()
    lib().orc_solve(ctypes.byref(prob.p), ctypes.byref(r))
    out = _result(r)
    tr = prob._trace
    # LTL_BS progress lines: (cost, op, AllLTLs, StoredLTLs, ToBeChecked)
    out["launches"] = [(int(tr[5 * i]), "~&|XFGUA"[tr[5 * i + 1]], int(tr[5 * i + 2]),
                        int(tr[5 * i + 3]), int(tr[5 * i + 4])) for i in range(r.trace_len)]
    return out


def solve_bs(prob: Problem, bs_max: int) -> dict:
    """solve(), then the BS stage up to size bs_max when nothing was found."""
    r = _Result()
    lib().orc_solve_bs(ctypes.byref(prob.p), bs_max, ctypes.byref(r))
    return _result(r)


def exhaustive(prob: Problem, max_formulas: int = 1 << 26) -> dict:
    r = _Result()
    lib().orc_exhaustive(ctypes.byref(prob.p), max_formulas, ctypes.byref(r))
    return _result(r)


def _encode(rpn):
    out = []
    for tk in rpn:
        out.append(tk if isinstance(tk, int) else -(1 + OPS.index(tk)))
    return out


def eval_rpn(prob: Problem, rpn) -> tuple[int, list[int]]:
    enc = _encode(rpn)
    arr = (ctypes.c_int16 * max(1, len(enc)))(*enc)
    cs = (ctypes.c_uint64 * prob.p.num_traces)()
    ok = lib().orc_eval_rpn(ctypes.byref(prob.p), arr, len(enc), cs)
    return ok, list(cs)


def make_key(prob: Problem, cs) -> tuple[int, int]:
    arr = (ctypes.c_uint64 * prob.p.num_traces)(*cs)
    h, l = ctypes.c_uint64(), ctypes.c_uint64()
    lib().orc_make_key(ctypes.byref(prob.p), arr, ctypes.byref(h), ctypes.byref(l))
    return h.value, l.value


def apply(prob: Problem, op: str, left, right=None) -> list[int]:
    t = prob.p.num_traces
    la = (ctypes.c_uint64 * t)(*left)
    ra = (ctypes.c_uint64 * t)(*(right if right is not None else [0] * t))
    out = (ctypes.c_uint64 * t)()
    lib().orc_apply(ctypes.byref(prob.p), OPS.index(op), la, ra, out)
    return list(out)


def ref_temp_capacity(prob: Problem) -> int:
    return lib().orc_ref_temp_capacity(ctypes.byref(prob.p))


def timed_solve(prob: Problem) -> tuple[dict, float]:
    t0 = time.perf_counter()
    res = solve(prob)
    return res, time.perf_counter() - t0
