"""The header-only C++ mirror (include/b200dedup_tree.hpp) builds against the C ABI, and the
ports of the reference's own ctest programs pass through it on the GPU."""
import json
import os
import subprocess

import pytest

from reproducibility_icpp23_scalable_gpu_deduplication_b200 import _build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "tree_tests.cpp")
BIN = os.path.join(ROOT, "tests", "cpp", "tree_tests")


def build_cpp():
    _build.build()
    pkg = os.path.dirname(_build.LIB_PATH)
    cmd = ["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"), "-I", "/usr/local/cuda/include", SRC,
           "-o", BIN, "-L", pkg, "-lb200dedup", f"-Wl,-rpath,{pkg}", "-L", "/usr/local/cuda/lib64", "-lcudart",
           "-Wl,-rpath,/usr/local/cuda/lib64"]
    subprocess.run(cmd, check=True)
    return BIN


def test_cpp_mirror_compiles():
    assert os.path.exists(build_cpp())


@pytest.mark.gpu
def test_cpp_reference_test_cases(cuda):
    b = build_cpp()
    with open(os.path.join(ROOT, "tests", "golden", "test_cases.json")) as f:
        cases = json.load(f)
    for k, c in sorted(cases.items()):
        r = subprocess.run([b, "case", c["step0"], c["step1"], str(c["first"]), str(c["shift"])],
                           capture_output=True, text=True)
        assert r.returncode == 0, (k, r.stdout, r.stderr)


@pytest.mark.gpu
@pytest.mark.parametrize("cs", [128, 64, 4096])
def test_cpp_tree_chkpt(cuda, cs):
    r = subprocess.run([build_cpp(), "tree_chkpt", str(cs), "10"], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("cs", [128, 64, 4096])
def test_cpp_list_chkpt(cuda, cs):
    """test/list_chkpt.cpp of the reference through b2d::ListDeduplicator"""
    r = subprocess.run([build_cpp(), "list_chkpt", str(cs), "10"], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr


@pytest.mark.gpu
def test_cpp_checkpoint_batch(cuda):
    r = subprocess.run([build_cpp(), "batch", "9"], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr


def test_cpp_sources_warning_free(tmp_path):
    """the C++ mirror, the ported reference tests and the file tools compile with -Wall -Wextra
    as errors (the mirror also with -pedantic)"""
    inc = ["-I", os.path.join(ROOT, "include"), "-I", "/usr/local/cuda/include"]
    hdr = tmp_path / "hdr.cpp"
    hdr.write_text('#include "b200dedup_tree.hpp"\nint main() { return 0; }\n')
    base = ["g++", "-std=c++17", "-Wall", "-Wextra", "-Werror", "-fsyntax-only"] + inc
    subprocess.run(base + ["-pedantic", str(hdr)], check=True)
    cli = os.path.join(ROOT, "reproducibility_icpp23_scalable_gpu_deduplication_b200", "cli")
    for src in [SRC] + sorted(os.path.join(cli, f) for f in os.listdir(cli) if f.endswith(".cpp")):
        subprocess.run(base + [src], check=True)
