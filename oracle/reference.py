"""Builds and drives the reference's own programs -- TEST INFRASTRUCTURE ONLY.

build_if_present() compiles the reference's sources, where they lie, into
oracle/_ref/ (never copied into this repository):

  ltl_nocache   nvcc ltl_nocache.cu -arch=sm_100a -std=c++20          (Makefile:4, retargeted)
  ltl_bs        nvcc LTL_BS.cu -I modified_libraries --extended-lambda  -arch=sm_100a -std=c++20

Both need a GPU to run; they are run only by tests/golden/make_goldens.py on a
B200 machine to produce the committed golden fixtures.  This module also holds
the JSON -> LTL_BS text converter (the format read by readFile,
LTL_BS.cu:1535-1607) and the parsers of both programs' output.
"""
from __future__ import annotations

import os
import re
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
NOCACHE = os.path.join(REF_DIR, "ltl_nocache")
LTL_BS = os.path.join(REF_DIR, "ltl_bs")
LTL_BS_TIMED = os.path.join(REF_DIR, "ltl_bs_timed")   # built with -DMEASUREMENT_MODE
# The reference checkout: VFB_REFERENCE_SRC, else a directory named
# "reference" beside this repository's root.
DEFAULT_SRC = os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference")


def build_if_present(src: str | None = None, force: bool = False) -> bool:
    """Compile the reference programs from the sources in `src` (default:
    VFB_REFERENCE_SRC, else DEFAULT_SRC) if they are there."""
    src = src or os.environ.get("VFB_REFERENCE_SRC") or DEFAULT_SRC
    if not os.path.exists(os.path.join(src, "LTL_BS.cu")):
        return False
    os.makedirs(REF_DIR, exist_ok=True)
    jobs = []
    if force or not os.path.exists(NOCACHE):
        jobs.append(["nvcc", os.path.join(src, "ltl_nocache.cu"), "-I", src, "-o", NOCACHE,
                     "-arch=sm_100a", "-std=c++20"])
    if force or not os.path.exists(LTL_BS):
        jobs.append(["nvcc", os.path.join(src, "LTL_BS.cu"), "-I",
                     os.path.join(src, "modified_libraries"), "--extended-lambda", "-o", LTL_BS,
                     "-arch=sm_100a", "-std=c++20"])
    if force or not os.path.exists(LTL_BS_TIMED):
        # the same program with its timing output (Running Time, Cost of Final
        # LTL; LTL_BS.cu:1661-1671, 1706-1710) in place of the progress lines
        jobs.append(["nvcc", os.path.join(src, "LTL_BS.cu"), "-I",
                     os.path.join(src, "modified_libraries"), "--extended-lambda", "-o", LTL_BS_TIMED,
                     "-arch=sm_100a", "-std=c++20", "-DMEASUREMENT_MODE"])
    procs = [subprocess.Popen(j, stdout=subprocess.PIPE, stderr=subprocess.STDOUT) for j in jobs]
    ok = True
    for p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            ok = False
            print(out.decode(errors="replace")[-4000:])
    return ok


def available() -> bool:
    return os.path.exists(NOCACHE) and os.path.exists(LTL_BS)


# ------------------------------------------------------------ LTL_BS text input
LETTERS = "abcdefghijklmnopqrstuvwxyz"


def instance_to_text(inst) -> str:
    """One line per trace: steps joined by ';', each step the propositions'
    0/1 values joined by ','; positives, '---', negatives, '---', then the
    alphabet line (propositions are renamed a, b, c, ... in order, so the
    reference's sorted alphabet keeps proposition order)."""
    if inst.num_vars > len(LETTERS):
        raise ValueError("LTL_BS reads at most 26 propositions (lowercase letters)")

    def line(length, words):
        return ";".join(",".join(str((words[v] >> t) & 1) for v in range(inst.num_vars))
                        for t in range(length))

    rows = [line(l, w) for l, w in inst.pos] + ["---"] + [line(l, w) for l, w in inst.neg]
    rows += ["---", ",".join(LETTERS[:inst.num_vars])]
    return "\n".join(rows) + "\n"


# ------------------------------------------------------------------- parsing
_BS_LINE = re.compile(r"Cost\s+(\d+)\s*\|\s*\((.)\)\s*\|\s*AllLTLs:\s*(\d+)\s*\|\s*StoredLTLs:\s*(\d+)"
                      r"\s*\|\s*ToBeChecked:\s*(\d+)")


def parse_ltl_bs(stdout: str) -> dict:
    """Launch log (cost, op, AllLTLs, StoredLTLs, ToBeChecked) and the formula."""
    launches = [(int(m.group(1)), m.group(2), int(m.group(3)), int(m.group(4)), int(m.group(5)))
                for m in _BS_LINE.finditer(stdout)]
    m = re.search(r'LTL: "(.*)"', stdout)
    return {"launches": launches, "formula": m.group(1) if m else None}


def parse_nocache(stdout: str, path: str) -> str | None:
    prefix = f"{path}, "
    for line in stdout.splitlines():
        if line.startswith(prefix):
            return line[len(prefix):]
    return None


def run_nocache(json_path: str, max_size: int, timeout: float = 600) -> dict:
    out = subprocess.run([NOCACHE, json_path, str(max_size)], capture_output=True, text=True,
                         timeout=timeout)
    return {"returncode": out.returncode, "formula": parse_nocache(out.stdout, json_path),
            "stderr_tail": out.stderr[-2000:]}


def run_ltl_bs(txt_path: str, max_size: int, rlx_type: int = 3, timeout: float = 600) -> dict:
    args = [LTL_BS, txt_path] + ["1"] * 8 + [str(max_size), str(max_size), str(rlx_type), "1"]
    out = subprocess.run(args, capture_output=True, text=True, timeout=timeout)
    res = parse_ltl_bs(out.stdout)
    res["returncode"] = out.returncode
    return res


def run_ltl_bs_timed(txt_path: str, max_size: int, rlx_type: int = 3, timeout: float = 300,
                     env: dict | None = None) -> dict:
    """One run of the timed LTL_BS build with unit costs and no BS stage:
    its own Running Time (the LTLI call, LTL_BS.cu:1661-1671), the final
    cost and the formula."""
    args = [LTL_BS_TIMED, txt_path] + ["1"] * 8 + [str(max_size), str(max_size), str(rlx_type), "1"]
    out = subprocess.run(args, capture_output=True, text=True, timeout=timeout, env=env)
    t = re.search(r"Running Time:\s*([0-9.eE+-]+)\s*s", out.stdout)
    c = re.search(r"Cost of Final LTL:\s*(-?\d+)", out.stdout)
    n = re.search(r"Number of All LTLs:\s*(\d+)", out.stdout)
    f = re.search(r'LTL: "(.*)"', out.stdout)
    return {"returncode": out.returncode, "seconds": float(t.group(1)) if t else None,
            "cost": int(c.group(1)) if c else None, "all_ltls": int(n.group(1)) if n else None,
            "formula": f.group(1) if f else None}


def timed_available() -> bool:
    return os.path.exists(LTL_BS_TIMED)


# ----------------------------------------------- formula text -> RPN tokens
def parse_infix(text: str, names) -> list:
    """Parse either notation ("(l) & (r)" of ltl_nocache or "(l)&(r)" of LTL_BS)
    into RPN tokens (proposition indices and operator characters)."""
    idx = {n: i for i, n in enumerate(names)}
    s = text.replace(" ", "")
    pos = 0

    def atom_or_group():
        nonlocal pos
        if s[pos] == "(":
            pos += 1
            r = expr()
            assert s[pos] == ")", (s, pos)
            pos += 1
            return r
        if s[pos] in "~XFG" and pos + 1 < len(s) and s[pos + 1] == "(":
            op = s[pos]
            pos += 2
            r = expr()
            assert s[pos] == ")"
            pos += 1
            return r + [op]
        # proposition name: longest match
        for n in sorted(idx, key=len, reverse=True):
            if s.startswith(n, pos):
                pos += len(n)
                return [idx[n]]
        raise ValueError(f"cannot parse at {pos}: {s}")

    def expr():
        nonlocal pos
        left = atom_or_group()
        if pos < len(s) and s[pos] in "&|U":
            op = s[pos]
            pos += 1
            right = atom_or_group()
            return left + right + [op]
        return left

    out = expr()
    if pos != len(s):
        raise ValueError(f"trailing text in {text!r}")
    return out
