"""Builds libb200dedup.so in-tree with nvcc for sm_100a (no JIT cache, no torch extension).

    python -m reproducibility_icpp23_scalable_gpu_deduplication_b200._build [--force]
"""
import os
import subprocess
import sys

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(PKG_DIR, "csrc")
LIB_PATH = os.path.join(PKG_DIR, "libb200dedup.so")
SOURCES = ["leaf.cu", "forest.cu", "gather.cu", "restart.cu", "dedup_host.cu", "batch.cu", "restart_noalloc.cu"]
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-shared",
]


def _nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def sources():
    return [os.path.join(CSRC, s) for s in SOURCES if os.path.exists(os.path.join(CSRC, s))]


def _stale():
    if not os.path.exists(LIB_PATH):
        return True
    t = os.path.getmtime(LIB_PATH)
    deps = sources() + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    deps.append(os.path.join(PKG_DIR, "..", "include", "b200dedup.h"))
    return any(os.path.getmtime(p) > t for p in deps if os.path.exists(p))


CLI_DIR = os.path.join(PKG_DIR, "cli")
INCLUDE = os.path.join(PKG_DIR, "..", "include")
# argv-compatible drivers of the reference's checkpoint-file tools, linked against the library
TOOLS = {"dedup_files": "dedup_files.cpp", "restart_chkpt_files": "restart_chkpt_files.cpp"}


def tool_path(name):
    return os.path.join(PKG_DIR, name)


def build_tools(force=False, verbose=False):
    for name, src in TOOLS.items():
        out, srcp = tool_path(name), os.path.join(CLI_DIR, src)
        deps = [srcp, LIB_PATH, os.path.join(INCLUDE, "b200dedup.h"), os.path.join(INCLUDE, "b200dedup_tree.hpp")]
        if not force and os.path.exists(out) and all(os.path.getmtime(d) <= os.path.getmtime(out) for d in deps):
            continue
        cmd = [_nvcc(), "-O2", "-std=c++17", "-Wno-deprecated-gpu-targets", "-I", INCLUDE, "-o", out + ".tmp", srcp, "-L", PKG_DIR, "-lb200dedup",
               "-Xlinker", "-rpath", "-Xlinker", "$ORIGIN"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True, cwd=CLI_DIR)
        os.replace(out + ".tmp", out)


def build(force=False, verbose=False):
    if force or _stale():
        tmp = LIB_PATH + ".tmp"
        cmd = [_nvcc()] + NVCC_FLAGS + ["-o", tmp] + sources()
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True, cwd=CSRC)
        os.replace(tmp, LIB_PATH)
    build_tools(force, verbose)
    return LIB_PATH


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
