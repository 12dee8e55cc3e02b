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
    # the list approach's constructor and the device-diff log writer check the same way
    assert L.b2d_create_list(0, 0, ctypes.byref(h)) == -1
    assert L.b2d_create_list(128, 7, ctypes.byref(h)) == -1
    assert L.b2d_write_chkpt_log(None, b"log") == -1
    assert L.b2d_copy_diff_async(None, None, 0, None) == -1
    assert L.b2d_restart_noalloc(None, 0, None, None, 0, 0, None) == -1


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


def test_host_digest_matches_reference_vectors():
    """b2d_hash_host (the library's own Murmur3 variant and MD5, run on the host) against the
    digests the reference's hash headers produced (tests/golden/hash_kat.json)"""
    import json

    with open(os.path.join(ROOT, "tests", "golden", "hash_kat.json")) as f:
        kat = json.load(f)["kat"]
    L = _lib.lib()
    out = ctypes.create_string_buffer(16)
    for e in kat:
        data = bytes.fromhex(e["data"])
        buf = ctypes.create_string_buffer(data, max(1, len(data)))
        for kind, key in ((_lib.HASH_MURMUR3, "murmur3"), (_lib.HASH_MD5, "md5")):
            assert L.b2d_hash_host(kind, buf, len(data), out) == 0
            assert out.raw.hex() == e[key], (key, e["len"])
    assert L.b2d_hash_host(7, buf, 1, out) != 0


def test_file_tools_build_and_check_arguments():
    """the argv-compatible file tools build with the library and reject what is not built here
    before touching a GPU"""
    _build.build()
    for name in _build.TOOLS:
        assert os.path.exists(_build.tool_path(name))
    r = subprocess.run([_build.tool_path("dedup_files")], capture_output=True, text=True)
    assert r.returncode == 1 and "usage" in r.stderr
    r = subprocess.run([_build.tool_path("dedup_files"), "128", "1", "--run-basic-chkpt", "x"],
                       capture_output=True, text=True)
    assert r.returncode == 2 and "only --run-tree-chkpt and --run-list-chkpt" in r.stderr
    r = subprocess.run([_build.tool_path("restart_chkpt_files"), "0", "1", "1", "128", "--run-full-chkpt", "x"],
                       capture_output=True, text=True)
    assert r.returncode == 2


def test_server_rejects_unknown_approach():
    """the served loop builds tree or list handles; any other approach is an argument error"""
    from reproducibility_icpp23_scalable_gpu_deduplication_b200.serve import CheckpointServer

    with pytest.raises(ValueError):
        CheckpointServer(approach="full")


def test_status_codes_match_header():
    """the Python status table names every code the C header declares, and the library has a
    message for each"""
    with open(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include",
                           "b200dedup.h")) as f:
        text = f.read()
    declared = {int(v): k for k, v in re.findall(r"\b(B2D_(?:OK|ERR_\w+))\s*=\s*(-?\d+)", text)}
    assert declared == _lib.STATUS
    L = _lib.lib()
    msgs = {code: L.b2d_strerror(code) for code in declared}
    assert all(msgs.values()) and len(set(msgs.values())) == len(msgs)


@pytest.mark.skipif(__import__("torch").cuda.is_available(), reason="checks the behaviour without a GPU")
def test_no_cpu_fallback_without_gpu():
    """without a CUDA device every entry point fails loudly: handles and batches cannot be
    created, and host tensors are refused before any call"""
    import torch

    from reproducibility_icpp23_scalable_gpu_deduplication_b200 import (B2DError, CheckpointBatch, ListDeduplicator,
                                                                        TreeDeduplicator)
    from reproducibility_icpp23_scalable_gpu_deduplication_b200.tree import hash_chunks

    for make in (lambda: TreeDeduplicator(128), lambda: ListDeduplicator(128), lambda: CheckpointBatch()):
        with pytest.raises(B2DError) as e:
            make()
        assert e.value.code == -2
    with pytest.raises(TypeError):
        hash_chunks(torch.zeros(256, dtype=torch.uint8), 128)


def test_header_is_plain_c(tmp_path):
    """include/b200dedup.h compiles as C99 and C11 with warnings as errors, and a C program that
    takes the address of every declared entry point links against the library"""
    _build.build()
    syms = header_symbols()
    src = tmp_path / "abi.c"
    src.write_text('#include "b200dedup.h"\n#include <stdio.h>\n'
                   "typedef void (*fp)(void);\n"
                   "int main(void) {\n  fp table[] = {\n"
                   + "".join(f"    (fp){s},\n" for s in syms)
                   + "  };\n  printf(\"%d %s\\n\", (int)(sizeof table / sizeof table[0]), b2d_strerror(0));\n"
                   "  return 0;\n}\n")
    pkg = os.path.dirname(_build.LIB_PATH)
    inc = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include")
    for std in ("c99", "c11"):
        exe = tmp_path / f"abi_{std}"
        subprocess.run(["gcc", f"-std={std}", "-Wall", "-Wextra", "-pedantic", "-Werror", "-I", inc, str(src),
                        "-o", str(exe), "-L", pkg, "-lb200dedup", f"-Wl,-rpath,{pkg}"], check=True)
        out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()
        assert out == [str(len(syms)), "ok"]
