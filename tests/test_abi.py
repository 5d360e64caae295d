"""CPU checks of the C ABI library: it loads, exports every symbol that
include/vfb.h declares, and its host-only entry points (JSON reader, infix
printer, CLI argument handling) behave like the reference's.  No GPU calls."""
import ctypes
import json
import os
import re
import subprocess

import pytest

import vfb_b200
from vfb_b200 import synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_symbols():
    syms = set()
    for name in os.listdir(os.path.join(ROOT, "include")):
        if name.endswith(".h"):
            text = open(os.path.join(ROOT, "include", name)).read()
            syms |= set(re.findall(r"\b(vfb_[a-z_]+)\s*\(", text))
    return syms


def test_library_exports_every_declared_symbol():
    lib = vfb_b200.load_library()
    syms = _declared_symbols()
    assert {"vfb_create", "vfb_solve", "vfb_batch_solve", "vfb_read_json"} <= syms
    for s in sorted(syms):
        assert hasattr(lib, s), s


def test_python_binding_lists_all_exports():
    assert set(vfb_b200.EXPORTS) <= _declared_symbols()


def test_struct_layouts_match_header(tmp_path):
    # sizes and field offsets of the ctypes mirrors equal the C compiler's
    src = tmp_path / "layout.c"
    src.write_text(
        '#include <stdio.h>\n#include <stddef.h>\n#include "vfb.h"\n'
        'int main(void) {\n'
        '  printf("%zu %zu %zu %zu %zu\\n", sizeof(vfb_tune), offsetof(vfb_tune, blocks),\n'
        '         offsetof(vfb_tune, ms), offsetof(vfb_tune, levels), sizeof(vfb_result));\n'
        '  return 0;\n}\n')
    exe = tmp_path / "layout"
    subprocess.check_call(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)])
    got = [int(x) for x in subprocess.check_output([str(exe)], text=True).split()]
    T = vfb_b200._Tune
    assert got == [ctypes.sizeof(T), T.blocks.offset, T.ms.offset, T.levels.offset,
                   ctypes.sizeof(vfb_b200._Result)]


def test_status_strings():
    lib = vfb_b200.load_library()
    assert lib.vfb_status_str(0) == b"ok"
    assert lib.vfb_status_str(1) == b"not found"


def _write(tmp_path, obj, name="t.json"):
    p = tmp_path / name
    p.write_text(json.dumps(obj) if not isinstance(obj, str) else obj)
    return str(p)


def test_read_json_matches_reference_encoding(tmp_path):
    inst = synth.config_planted()
    path = _write(tmp_path, inst.to_json())
    prob = vfb_b200.read_json_file(path)
    ref = vfb_b200.Problem.from_instance(inst)
    assert prob.num_vars == ref.num_vars and prob.num_pos == ref.num_pos
    assert prob.words == ref.words and prob.lengths == ref.lengths
    assert prob.names == ref.names


def test_read_json_length_from_first_proposition(tmp_path):
    d = {"number_atomic_propositions": 2, "number_traces": 2, "number_positive_traces": 1,
         "max_length_traces": 5, "atomic_propositions": ["x", "y"],
         "positive_traces": [{"x": [1, 0, 1], "y": [0, 1, 1, 1, 1]}],
         "negative_traces": [{"y": [1], "x": [0, 1]}], "extra": {"ignored": [1, 2]}}
    prob = vfb_b200.read_json_file(_write(tmp_path, d))
    assert prob.lengths == [3, 2]
    # bits past the first proposition's length are kept, as in the reference
    assert prob.words == [0b101, 0b11110, 0b10, 0b1]


@pytest.mark.parametrize("bad", [
    "{", "[]", '{"number_atomic_propositions": 1}',
    {"number_atomic_propositions": 1, "number_traces": 2, "number_positive_traces": 1,
     "max_length_traces": 2, "atomic_propositions": ["a"],
     "positive_traces": [{"a": [1]}], "negative_traces": []},
    {"number_atomic_propositions": 1, "number_traces": 1, "number_positive_traces": 1,
     "max_length_traces": 65, "atomic_propositions": ["a"],
     "positive_traces": [{"a": [1] * 65}], "negative_traces": []},
    {"number_atomic_propositions": 2, "number_traces": 1, "number_positive_traces": 1,
     "max_length_traces": 2, "atomic_propositions": ["a", "b"],
     "positive_traces": [{"a": [1, 0]}], "negative_traces": []},
])
def test_read_json_rejects_malformed(tmp_path, bad):
    with pytest.raises(vfb_b200.VfbError):
        vfb_b200.read_json_file(_write(tmp_path, bad))


def test_read_json_missing_file():
    with pytest.raises(vfb_b200.VfbError, match="Could not open file"):
        vfb_b200.read_json_file("/nonexistent/none.json")


def test_format_infix_reference_notation():
    lib = vfb_b200.load_library()
    r = vfb_b200._Result()
    toks = [0, -4, -1, 1, -7, 0, -6, -3]     # ((~(X(a))) U (b)) | (G(a))
    r.rpn_len = len(toks)
    for i, t in enumerate(toks):
        r.rpn[i] = t
    names = (ctypes.c_char_p * 2)(b"a", b"b")
    buf = ctypes.create_string_buffer(256)
    n = lib.vfb_format_infix(ctypes.byref(r), names, buf, 256)
    text = buf.value.decode()
    assert text == "((~(X(a))) U (b)) | (G(a))"
    assert n == len(text)
    res = vfb_b200.Result(0, 8, [0, "X", "~", 1, "U", 0, "G", "|"], [], [], 0, 0, 0.0)
    assert res.infix(["a", "b"]) == text
    assert synth.rpn_to_infix([0, "X", "~", 1, "U", 0, "G", "|"], ["a", "b"]) == text


def test_format_infix_rejects_malformed():
    lib = vfb_b200.load_library()
    r = vfb_b200._Result()
    r.rpn_len = 2
    r.rpn[0] = 0
    r.rpn[1] = -2          # binary op with one operand
    assert lib.vfb_format_infix(ctypes.byref(r), None, None, 0) == -1


def _cli(*args):
    return subprocess.run([vfb_b200.CLI_PATH, *args], capture_output=True, text=True, timeout=60)


def test_cli_usage_and_argument_errors(tmp_path):
    out = _cli()
    assert out.returncode == 0 and out.stdout == ""
    assert "<input_file_address> <maxLen>" in out.stderr
    out = _cli("x.json", "0")
    assert out.returncode == 0 and "should be between 1 and 32" in out.stderr
    out = _cli("x.json", "51")
    assert out.returncode == 0 and "should be between 1 and 32" in out.stderr
    path = _write(tmp_path, synth.config_small().to_json())
    out = _cli(path, "40")
    assert out.returncode == 0 and out.stderr == "This version supports formulas of size at most 32.\n"
    out = _cli("/nonexistent.json", "5")
    assert out.returncode == 0 and "Could not open file" in out.stderr


def test_cli_strict_exit_codes():
    out = _cli("--strict-exit")
    assert out.returncode == 2


def test_problem_c_arrays_follow_assignment():
    # the C arrays are converted once per Problem; assigning new words or
    # lengths converts again, and the scalar fields are read at every call
    prob = vfb_b200.Problem.from_instance(synth.config_planted())
    s1, keep1 = prob._cstruct()
    assert list(keep1[0]) == prob.words and list(keep1[1]) == prob.lengths
    assert [s1.words[i] for i in range(len(prob.words))] == prob.words
    s1b, keep1b = prob._cstruct()
    assert keep1b[0] is keep1[0]
    prob.words = [w ^ 1 for w in prob.words]
    s2, keep2 = prob._cstruct()
    assert keep2[0] is not keep1[0]
    assert [s2.words[i] for i in range(len(prob.words))] == prob.words
    prob.lengths = list(prob.lengths)
    prob.max_size = 3
    s3, keep3 = prob._cstruct()
    assert keep3[1] is not keep2[1] and s3.max_size == 3 and s3.num_traces == len(prob.lengths)


def test_problem_pickles_after_a_conversion():
    import copy
    import pickle
    prob = vfb_b200.Problem.from_instance(synth.config_planted())
    prob._cstruct()
    again = pickle.loads(pickle.dumps(prob))
    assert again == prob and copy.deepcopy(prob) == prob
    s, keep = again._cstruct()
    assert [s.words[i] for i in range(len(again.words))] == again.words
