"""The C-ABI library loads and exports every function include/prism_solve.h declares."""
from __future__ import annotations

import os
import re
import subprocess

import prispack_b200 as P

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def declared():
    src = open(os.path.join(ROOT, "include", "prism_solve.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(prism_[a-z0-9_]+)\s*\(", src)))


def test_header_declarations_are_exported():
    lib = P.load()
    names = declared()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    assert sorted(P.exported_symbols()) == declared()


def test_dynamic_symbol_table():
    out = subprocess.run(["nm", "-D", "--defined-only", P.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (prism_[a-z0-9_]+)", out))
    assert set(declared()) <= exported


def test_build_targets_sm100a_only():
    from prispack_b200 import build
    assert build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]


def test_last_error_and_version():
    lib = P.load()
    assert lib.prism_version() >= 100
    # a host-side argument error leaves a message
    import ctypes as C
    n = C.c_uint32()
    rc = lib.prism_laplacian_dims(0, 1, 1, C.byref(n), C.byref(C.c_uint32()))
    assert rc == 1 and b"range" in lib.prism_last_error()
