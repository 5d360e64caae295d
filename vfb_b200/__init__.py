"""vfb_b200 -- B200-native bottom-up LTL formula learning (VFB's cached search).

Python host-side binding of the C ABI in include/vfb.h (libvfb_b200.so).  The
entry points mirror the reference's host interface:

  ltl(max_len, input_data, trace_len, num_vars, num_pos, names)
      -> the formula string, "Not found !" or raises; same arguments and
         meaning as std::string LTL(maxLen, inputData, traceLen, traceLength)
         of ltl_nocache.cu:319 (whose inputs are globals there).
  read_json_file(path) -> Problem       (readJsonFile, ltl_nocache.cu:35-76)
  Engine.solve / Engine.batch_solve     (vfb_solve / vfb_batch_solve)

The search itself runs only in the CUDA library: there is no CPU fallback, and
importing the engine on a machine without the built library or a B200 raises.
"""
from __future__ import annotations

import array
import ctypes
import os
import threading
from dataclasses import dataclass, field

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libvfb_b200.so")
CLI_PATH = os.path.join(HERE, "_lib", "vfb")
OPS = "~&|XFGU"
MAX_SIZE = 32

OK, NOT_FOUND, LIMIT, OOM, DEVICE_ERROR, TIMEOUT, BAD_INPUT = range(7)
STATUS_NAMES = ["ok", "not found", "limit", "oom", "device error", "timeout", "bad input"]


class VfbError(RuntimeError):
    pass


class _Opts(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("mem_limit_bytes", ctypes.c_size_t),
                ("verbose", ctypes.c_int), ("profile", ctypes.c_int)]


class _Instance(ctypes.Structure):
    _fields_ = [("num_vars", ctypes.c_int), ("num_traces", ctypes.c_int),
                ("num_pos", ctypes.c_int), ("words", ctypes.POINTER(ctypes.c_uint64)),
                ("lengths", ctypes.POINTER(ctypes.c_int)), ("max_size", ctypes.c_int),
                ("rlx_type", ctypes.c_int)]


_P_U64 = ctypes.POINTER(ctypes.c_uint64)
_P_INT = ctypes.POINTER(ctypes.c_int)


class _Result(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("size", ctypes.c_int), ("rpn_len", ctypes.c_int),
                ("rpn", ctypes.c_int16 * MAX_SIZE),
                ("level_rows", ctypes.c_uint64 * (MAX_SIZE + 1)),
                ("level_cands", ctypes.c_uint64 * (MAX_SIZE + 1)),
                ("total_rows", ctypes.c_uint64), ("solution_index", ctypes.c_uint64),
                ("seconds", ctypes.c_double), ("device_seconds", ctypes.c_double),
                ("h2d_bytes", ctypes.c_uint64), ("d2h_bytes", ctypes.c_uint64),
                ("kernel_launches", ctypes.c_uint64)]


class _Served(ctypes.Structure):
    _fields_ = [("tag", ctypes.c_uint64), ("result", _Result)]


class _KernelStat(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char * 32), ("launches", ctypes.c_uint64),
                ("ms", ctypes.c_double), ("bytes", ctypes.c_double)]


TUNE_BANDS = 16


class _Tune(ctypes.Structure):
    _fields_ = [("rows", ctypes.c_uint8 * TUNE_BANDS), ("tiles_log2", ctypes.c_uint8 * TUNE_BANDS),
                ("blocks", ctypes.c_uint16 * TUNE_BANDS), ("ms", ctypes.c_float * TUNE_BANDS),
                ("ms_default", ctypes.c_float * TUNE_BANDS), ("levels", ctypes.c_uint32 * TUNE_BANDS)]


def _tune_dict(t: _Tune) -> dict:
    return {f: list(getattr(t, f)) for f, _ in _Tune._fields_}


class _JsonProblem(ctypes.Structure):
    _fields_ = [("inst", _Instance), ("max_length_traces", ctypes.c_int),
                ("names", ctypes.POINTER(ctypes.c_char_p))]


EXPORTS = ["vfb_create", "vfb_destroy", "vfb_solve", "vfb_batch_solve", "vfb_status_str",
           "vfb_read_json", "vfb_json_free", "vfb_format_infix", "vfb_profile_read",
           "vfb_profile_reset", "vfb_solve_noalloc", "vfb_synth_planted", "vfb_serve_open",
           "vfb_serve_limits", "vfb_serve_submit", "vfb_serve_step", "vfb_serve_close",
           "vfb_solve_exhaustive", "vfb_solve_bs", "vfb_solve_costs", "vfb_tune_set",
           "vfb_tune_get", "vfb_autotune"]

_lib = None


def load_library():
    """Load libvfb_b200.so (building it first if the sources are newer)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        try:
            from . import build as _build
            _build.build()
        except Exception as e:  # noqa: BLE001
            raise VfbError(f"libvfb_b200.so is missing and could not be built: {e}") from e
    lib = ctypes.CDLL(LIB_PATH)
    lib.vfb_create.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(_Opts)]
    lib.vfb_create.restype = ctypes.c_int
    lib.vfb_destroy.argtypes = [ctypes.c_void_p]
    lib.vfb_destroy.restype = None
    lib.vfb_solve.argtypes = [ctypes.c_void_p, ctypes.POINTER(_Instance), ctypes.POINTER(_Result)]
    lib.vfb_solve.restype = ctypes.c_int
    lib.vfb_batch_solve.argtypes = [ctypes.c_void_p, ctypes.POINTER(_Instance), ctypes.c_int,
                                    ctypes.POINTER(_Result)]
    lib.vfb_batch_solve.restype = ctypes.c_int
    lib.vfb_status_str.argtypes = [ctypes.c_int]
    lib.vfb_status_str.restype = ctypes.c_char_p
    lib.vfb_read_json.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.POINTER(_JsonProblem)),
                                  ctypes.c_char_p, ctypes.c_size_t]
    lib.vfb_read_json.restype = ctypes.c_int
    lib.vfb_json_free.argtypes = [ctypes.POINTER(_JsonProblem)]
    lib.vfb_json_free.restype = None
    lib.vfb_format_infix.argtypes = [ctypes.POINTER(_Result), ctypes.POINTER(ctypes.c_char_p),
                                     ctypes.c_char_p, ctypes.c_size_t]
    lib.vfb_format_infix.restype = ctypes.c_int
    lib.vfb_profile_read.argtypes = [ctypes.c_void_p, ctypes.POINTER(_KernelStat), ctypes.c_int]
    lib.vfb_profile_read.restype = ctypes.c_int
    lib.vfb_profile_reset.argtypes = [ctypes.c_void_p]
    lib.vfb_profile_reset.restype = None
    lib.vfb_solve_noalloc.argtypes = [ctypes.POINTER(_Instance), ctypes.POINTER(_Result)]
    lib.vfb_solve_noalloc.restype = ctypes.c_int
    lib.vfb_serve_open.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
    lib.vfb_serve_open.restype = ctypes.c_int
    lib.vfb_solve_costs.argtypes = [ctypes.c_void_p, ctypes.POINTER(_Instance), ctypes.POINTER(ctypes.c_int),
                                     ctypes.c_int, ctypes.POINTER(_Result)]
    lib.vfb_solve_costs.restype = ctypes.c_int
    lib.vfb_solve_bs.argtypes = [ctypes.c_void_p, ctypes.POINTER(_Instance), ctypes.c_int, ctypes.POINTER(_Result)]
    lib.vfb_solve_bs.restype = ctypes.c_int
    lib.vfb_solve_exhaustive.argtypes = [ctypes.c_void_p, ctypes.POINTER(_Instance), ctypes.POINTER(_Result)]
    lib.vfb_solve_exhaustive.restype = ctypes.c_int
    lib.vfb_serve_limits.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_uint64, ctypes.c_uint64]
    lib.vfb_serve_limits.restype = ctypes.c_int
    lib.vfb_serve_submit.argtypes = [ctypes.c_void_p, ctypes.POINTER(_Instance), ctypes.c_uint64]
    lib.vfb_serve_submit.restype = ctypes.c_int
    lib.vfb_serve_step.argtypes = [ctypes.c_void_p, ctypes.POINTER(_Served), ctypes.c_int,
                                   ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                   ctypes.POINTER(ctypes.c_int)]
    lib.vfb_serve_step.restype = ctypes.c_int
    lib.vfb_serve_close.argtypes = [ctypes.c_void_p]
    lib.vfb_serve_close.restype = None
    lib.vfb_tune_set.argtypes = [ctypes.c_void_p, ctypes.POINTER(_Tune)]
    lib.vfb_tune_set.restype = ctypes.c_int
    lib.vfb_tune_get.argtypes = [ctypes.c_void_p, ctypes.POINTER(_Tune)]
    lib.vfb_tune_get.restype = ctypes.c_int
    lib.vfb_autotune.argtypes = [ctypes.c_void_p, ctypes.POINTER(_Instance), ctypes.c_int, ctypes.c_int,
                                 ctypes.POINTER(_Tune)]
    lib.vfb_autotune.restype = ctypes.c_int
    _lib = lib
    return lib


# ------------------------------------------------------------------- problems
@dataclass
class Problem:
    """Inputs in the reference's layout: words[i*num_vars + v], lengths[i]."""
    num_vars: int
    num_pos: int
    words: list
    lengths: list
    names: list = field(default_factory=list)
    max_size: int = MAX_SIZE
    rlx_type: int = 3
    max_length_traces: int = 0

    @property
    def num_traces(self) -> int:
        return len(self.lengths)

    @classmethod
    def from_instance(cls, inst) -> "Problem":
        """From a vfb_b200.synth.Instance."""
        traces = inst.pos + inst.neg
        words = [w[v] for _, w in traces for v in range(inst.num_vars)]
        return cls(inst.num_vars, len(inst.pos), words, [l for l, _ in traces],
                   list(inst.names) or [f"a{v}" for v in range(inst.num_vars)],
                   inst.max_size, inst.rlx_type, max(l for l, _ in traces))

    def __setattr__(self, name, value):
        # assigning new words or lengths drops the converted copies
        if name in ("words", "lengths"):
            object.__setattr__(self, "_arrays", None)
        object.__setattr__(self, name, value)

    def __getstate__(self):
        # (the converted copies hold C pointers: not pickled, rebuilt on use)
        state = dict(self.__dict__)
        state.pop("_arrays", None)
        return state

    def __setstate__(self, state):
        self.__dict__.update(state)

    def _cstruct(self):
        # the C arrays are Python array buffers, converted once per Problem
        # (words and lengths are taken as fixed once a Problem has been
        # solved: assign new lists to change them); the caller keeps them
        # alive until the call returns
        arrays = getattr(self, "_arrays", None)
        if arrays is None:
            w = array.array("Q", self.words or [0])
            ln = array.array("i", self.lengths or [0])
            arrays = (w, ln, ctypes.cast(w.buffer_info()[0], _P_U64), ctypes.cast(ln.buffer_info()[0], _P_INT))
            object.__setattr__(self, "_arrays", arrays)
        w, ln, wp, lp = arrays
        s = _Instance(self.num_vars, len(self.lengths), self.num_pos, wp, lp, self.max_size, self.rlx_type)
        return s, (w, ln)


@dataclass
class Result:
    status: int
    size: int
    rpn: list
    level_rows: list
    level_cands: list
    total_rows: int
    solution_index: int
    seconds: float
    device_seconds: float = 0.0
    h2d_bytes: int = 0
    d2h_bytes: int = 0
    kernel_launches: int = 0

    @property
    def found(self) -> bool:
        return self.status == OK

    def infix(self, names) -> str:
        st = []
        for tk in self.rpn:
            if isinstance(tk, int):
                st.append(names[tk])
            elif tk in "~XFG":
                st.append(f"{tk}({st.pop()})")
            else:
                r = st.pop()
                l = st.pop()
                st.append(f"({l}) {tk} ({r})")
        return st[0] if len(st) == 1 else ""


def _result(r: _Result) -> Result:
    k = max(0, min(r.size, MAX_SIZE))
    rpn = [x if x >= 0 else OPS[-x - 1] for x in r.rpn[:max(0, min(r.rpn_len, MAX_SIZE))]]
    return Result(r.status, r.size, rpn, r.level_rows[1:k + 1],
                  r.level_cands[1:k + 1], r.total_rows, r.solution_index,
                  r.seconds, r.device_seconds, r.h2d_bytes, r.d2h_bytes, r.kernel_launches)


def read_json_file(path: str) -> Problem:
    """Parse a trace file in the reference's JSON schema with the library's reader."""
    lib = load_library()
    out = ctypes.POINTER(_JsonProblem)()
    err = ctypes.create_string_buffer(512)
    rc = lib.vfb_read_json(path.encode(), ctypes.byref(out), err, len(err))
    if rc != OK:
        raise VfbError(err.value.decode() or STATUS_NAMES[rc])
    try:
        jp = out.contents
        inst = jp.inst
        t, a = inst.num_traces, inst.num_vars
        words = [inst.words[i] for i in range(t * a)]
        lengths = [inst.lengths[i] for i in range(t)]
        names = [jp.names[v].decode() for v in range(a)]
        return Problem(a, inst.num_pos, words, lengths, names, MAX_SIZE, 3, jp.max_length_traces)
    finally:
        lib.vfb_json_free(out)


# --------------------------------------------------------------------- engine
class Engine:
    """One CUDA context/stream of the engine (vfb_create ... vfb_destroy)."""

    def __init__(self, device: int = 0, mem_limit_bytes: int = 0, verbose: bool = False,
                 profile: bool = False):
        self._lib = load_library()
        self._ctx = ctypes.c_void_p()
        opts = _Opts(device, mem_limit_bytes, 1 if verbose else 0, 1 if profile else 0)
        rc = self._lib.vfb_create(ctypes.byref(self._ctx), ctypes.byref(opts))
        if rc != OK:
            raise VfbError(f"vfb_create failed: {STATUS_NAMES[rc]} (a B200 and the sm_100a build "
                           "are required; there is no CPU fallback)")

    def close(self):
        if self._ctx:
            self._lib.vfb_destroy(self._ctx)
            self._ctx = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001
            pass

    def profile(self) -> list:
        """Per-kernel (name, launches, total ms, algorithmic bytes) since creation."""
        arr = (_KernelStat * 32)()
        m = self._lib.vfb_profile_read(self._ctx, arr, 32)
        return [(arr[i].name.decode(), arr[i].launches, arr[i].ms, arr[i].bytes) for i in range(m)]

    def profile_reset(self) -> None:
        self._lib.vfb_profile_reset(self._ctx)

    def solve(self, prob: Problem) -> Result:
        inst, keep = prob._cstruct()
        res = _Result()
        self._lib.vfb_solve(self._ctx, ctypes.byref(inst), ctypes.byref(res))
        del keep
        return _result(res)

    def solve_costs(self, prob: Problem, costs, neg_type: int = 1) -> Result:
        """solve() with LTL_BS's operator costs [p, ~, &, |, X, F, G, U] and NegType;
        sizes in the result are then costs."""
        inst, keep = prob._cstruct()
        res = _Result()
        arr = (ctypes.c_int * 8)(*costs)
        self._lib.vfb_solve_costs(self._ctx, ctypes.byref(inst), arr, neg_type, ctypes.byref(res))
        del keep
        return _result(res)

    def solve_bs(self, prob: Problem, bs_max_size: int) -> Result:
        """solve(), then the BS stage up to bs_max_size when nothing was found."""
        inst, keep = prob._cstruct()
        res = _Result()
        self._lib.vfb_solve_bs(self._ctx, ctypes.byref(inst), bs_max_size, ctypes.byref(res))
        del keep
        return _result(res)

    def solve_exhaustive(self, prob: Problem) -> Result:
        """Cache-free search in formula-number order (the ltl_nocache method)."""
        inst, keep = prob._cstruct()
        res = _Result()
        self._lib.vfb_solve_exhaustive(self._ctx, ctypes.byref(inst), ctypes.byref(res))
        del keep
        return _result(res)

    # ---- k_p1 launch shape per level band
    def autotune(self, probs: list, reps: int = 2) -> dict:
        """Time k_p1 over the sample under each candidate shape and install the
        fastest per level band; returns the table (vfb_tune fields as lists)."""
        n = len(probs)
        arr = (_Instance * n)()
        keep = []
        for i, p in enumerate(probs):
            s, k = p._cstruct()
            arr[i] = s
            keep.append(k)
        t = _Tune()
        rc = self._lib.vfb_autotune(self._ctx, arr, n, reps, ctypes.byref(t))
        del keep
        if rc != OK:
            raise VfbError(f"vfb_autotune failed: {STATUS_NAMES[rc]}")
        return _tune_dict(t)

    def set_tune(self, table) -> None:
        """Install a shape table (dict with rows / tiles_log2 / blocks lists; None: built-in)."""
        if table is None:
            rc = self._lib.vfb_tune_set(self._ctx, None)
        else:
            t = _Tune()
            for f, _ in _Tune._fields_:
                if f in table:
                    getattr(t, f)[:] = list(table[f])
            rc = self._lib.vfb_tune_set(self._ctx, ctypes.byref(t))
        if rc != OK:
            raise VfbError(f"vfb_tune_set failed: {STATUS_NAMES[rc]}")

    def get_tune(self) -> dict:
        t = _Tune()
        self._lib.vfb_tune_get(self._ctx, ctypes.byref(t))
        return _tune_dict(t)

    # ---- serving (continuous batching)
    def serve_limits(self, budget_frac: float = 0.8, request_bytes: int = 0,
                     step_candidates: int = 1 << 23) -> None:
        """Admission fraction of the memory budget, per-request byte cap (0: budget / 4) and
        operator candidates of one request per step (0: whole levels)."""
        rc = self._lib.vfb_serve_limits(self._ctx, budget_frac, request_bytes, step_candidates)
        if rc != OK:
            raise VfbError(f"vfb_serve_limits failed: {STATUS_NAMES[rc]}")

    def serve_open(self, slots: int = 256, max_traces: int = 64) -> None:
        rc = self._lib.vfb_serve_open(self._ctx, slots, max_traces)
        if rc != OK:
            raise VfbError(f"vfb_serve_open failed: {STATUS_NAMES[rc]}")
        self._served = (_Served * max(slots, 64))()

    def serve_submit(self, prob: Problem, tag: int) -> None:
        inst, keep = prob._cstruct()
        rc = self._lib.vfb_serve_submit(self._ctx, ctypes.byref(inst), tag)
        del keep
        if rc != OK:
            raise VfbError(f"vfb_serve_submit failed: {STATUS_NAMES[rc]}")

    def serve_step(self):
        """One admission + level step; returns ([(tag, Result)], active, queued)."""
        nd, act, q = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        rc = self._lib.vfb_serve_step(self._ctx, self._served, len(self._served), ctypes.byref(nd),
                                      ctypes.byref(act), ctypes.byref(q))
        if rc != OK:
            raise VfbError(f"vfb_serve_step failed: {STATUS_NAMES[rc]}")
        done = [(self._served[i].tag, _result(self._served[i].result)) for i in range(nd.value)]
        return done, act.value, q.value

    def serve_close(self) -> None:
        self._lib.vfb_serve_close(self._ctx)

    def batch_solve(self, probs: list) -> list:
        n = len(probs)
        if n == 0:
            return []
        arr = (_Instance * n)()
        keep = []
        for i, p in enumerate(probs):
            s, k = p._cstruct()
            arr[i] = s
            keep.append(k)
        res = (_Result * n)()
        rc = self._lib.vfb_batch_solve(self._ctx, arr, n, res)
        if rc not in (OK, NOT_FOUND):
            raise VfbError(f"vfb_batch_solve failed: {STATUS_NAMES[rc]}")
        return [_result(res[i]) for i in range(n)]


_noalloc_lock = threading.Lock()


def solve_noalloc(prob: Problem) -> Result:
    """vfb_solve_noalloc: the solve without any allocation (static scratch of
    VFB_NOALLOC_SCRATCH_BYTES on the current device; VFB_OOM if it does not fit).

    Every call uses the same static device array, and the C call releases the
    GIL, so calls from several Python threads would race on it: they are
    serialised here by a module-level lock."""
    lib = load_library()
    inst, keep = prob._cstruct()
    res = _Result()
    with _noalloc_lock:
        lib.vfb_solve_noalloc(ctypes.byref(inst), ctypes.byref(res))
    del keep
    return _result(res)


def ltl(max_len: int, input_data, trace_len, num_vars: int, num_pos: int, names,
        rlx_type: int = 3, engine: Engine | None = None) -> str:
    """Same contract as the reference's LTL(): the smallest formula's infix text,
    or "Not found !" when none exists up to max_len."""
    eng = engine or Engine()
    res = eng.solve(Problem(num_vars, num_pos, list(input_data), list(trace_len), list(names),
                            max_len, rlx_type))
    if res.status == OK:
        return res.infix(names)
    if res.status == NOT_FOUND:
        return "Not found !"
    raise VfbError(STATUS_NAMES[res.status])
