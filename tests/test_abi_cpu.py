"""The C ABI library without a GPU: it loads, exports every function that
include/tritracer.h declares, and the ctypes mirrors of the argument structs
match the C layout (checked by compiling a probe against the header with gcc).
No compute call is made."""
import ctypes
import os
import re
import subprocess
import sys
import tempfile

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "tritracer.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(tt_\w+)\s*\(", src, flags=re.M)))


def test_header_declares_the_api():
    names = declared_functions()
    for n in ("tt_create", "tt_destroy", "tt_build", "tt_forward", "tt_backward", "tt_last_error"):
        assert n in names


def test_library_exports_every_declared_symbol():
    from diff_tritracer import _lib

    lib = ctypes.CDLL(_lib.LIB_PATH)
    for name in declared_functions():
        assert hasattr(lib, name), name
    assert set(_lib.EXPORTS) <= set(declared_functions())


def test_struct_layout_matches_header():
    from diff_tritracer import _lib

    structs = {"tt_config": _lib.TtConfig, "tt_fwd_args": _lib.TtFwdArgs, "tt_bwd_args": _lib.TtBwdArgs,
               "tt_view": _lib.TtView, "tt_stats": _lib.TtStats, "tt_mlp": _lib.TtMlp,
               "tt_mlp_step": _lib.TtMlpStep, "tt_secondary": _lib.TtSecondary, "tt_camera": _lib.TtCamera}
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', "int main(void){"]
    for cname, py in structs.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines.append("return 0;}")
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "probe.c")
        exe = os.path.join(d, "probe")
        open(c, "w").write("\n".join(lines))
        subprocess.run(["gcc", "-std=c99", c, "-o", exe], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {}
    for ln in out:
        if ln:
            s, f, v = ln.split()
            got[(s, f)] = int(v)
    for cname, py in structs.items():
        assert got[(cname, "size")] == ctypes.sizeof(py), cname
        for fname, _ in py._fields_:
            assert got[(cname, fname)] == getattr(py, fname).offset, (cname, fname)


def test_missing_library_fails_loudly(monkeypatch):
    from diff_tritracer import _lib

    monkeypatch.setattr(_lib, "LIB_PATH", "/nonexistent/libtritracer.so")
    with pytest.raises(ImportError, match="no CPU fallback"):
        _lib._load()


def test_oracle_intersector_known_answers(oracle):
    # ray along -z through a unit triangle in the z=0 plane, from z=3
    hit, t = oracle.isect([0.1, 0.1, 3.0], [0, 0, -1], [0, 0, 0], [1, 0, 0], [0, 1, 0])
    assert hit and t == pytest.approx(3.0)
    # the other winding hits too (non-culling)
    hit, t = oracle.isect([0.1, 0.1, 3.0], [0, 0, -1], [0, 0, 0], [0, 1, 0], [1, 0, 0])
    assert hit and t == pytest.approx(3.0)
    hit, _ = oracle.isect([1.1, 0.1, 3.0], [0, 0, -1], [0, 0, 0], [1, 0, 0], [0, 1, 0])
    assert not hit
