"""The C-ABI library loads and exports every symbol include/b200dedup.h declares (no GPU)."""
import ctypes
import os
import re
import subprocess

import pytest

from reproducibility_icpp23_scalable_gpu_deduplication_b200 import _build, _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    txt = open(os.path.join(ROOT, "include", "b200dedup.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(b2d_[a-z0-9_]+)\s*\(", txt)))


def test_library_builds_and_loads():
    path = _build.build()
    assert os.path.exists(path)
    assert _lib.lib() is not None


def test_exports_every_declared_symbol():
    syms = header_symbols()
    assert len(syms) >= 20
    out = subprocess.run(["nm", "-D", "--defined-only", _build.LIB_PATH], capture_output=True, text=True,
                         check=True).stdout
    exported = set(re.findall(r"\bT (b2d_\w+)", out))
    missing = [s for s in syms if s not in exported]
    assert not missing, missing
    # and the ctypes table binds exactly the declared set
    assert sorted(n for n, _, _ in _lib.SIGNATURES) == syms


def test_strerror_and_argument_errors_without_gpu():
    L = _lib.lib()
    assert L.b2d_strerror(0) == b"ok"
    assert L.b2d_strerror(-6) == b"digest map full"
    # invalid arguments are rejected before any device work
    h = ctypes.c_void_p()
    assert L.b2d_create(0, 0, ctypes.byref(h)) == -1
    assert L.b2d_create(128, 7, ctypes.byref(h)) == -1
    assert L.b2d_destroy(None) == -1
    v = ctypes.c_uint64()
    assert L.b2d_num_first_ocur(None, ctypes.byref(v)) == -1


def test_no_oracle_in_product():
    """The product library never links or loads the oracle."""
    out = subprocess.run(["ldd", _build.LIB_PATH], capture_output=True, text=True).stdout
    assert "oracle" not in out
    pkg = os.path.join(ROOT, "reproducibility_icpp23_scalable_gpu_deduplication_b200")
    for dirpath, _, files in os.walk(pkg):
        for f in files:
            if f.endswith((".py", ".cu", ".cuh", ".h", ".cpp")):
                txt = open(os.path.join(dirpath, f), errors="ignore").read()
                assert "import oracle" not in txt and "from oracle" not in txt, f
