"""Build the sm_100a library in-tree: fmm_gen_b200/lib/libfmm_b200.so.

    python -m fmm_gen_b200.build [--verbose]

nvcc cross-compiles without a GPU.  The library links the CUDA runtime statically,
so it loads into any process (torch included) without a matching libcudart.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB_DIR = os.path.join(PKG, "lib")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-shared"] + ARCH


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


SOURCES = ["fmm_capi.cu"]
HEADERS = ["fmm_kernels.cuh", "fmm_split_bf16.cuh", os.path.join("..", "..", "include", "fmm_b200.h")]


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(LIB_DIR, exist_ok=True)
    out = os.path.join(LIB_DIR, "libfmm_b200.so")
    deps = [os.path.join(CSRC, s) for s in SOURCES + HEADERS]
    if force or _stale(out, deps):
        cmd = [nvcc()] + NVCC_FLAGS + (["-Xptxas", "-v"] if verbose else []) + ["-o", out] + \
              [os.path.join(CSRC, s) for s in SOURCES]
        subprocess.run(cmd, check=True)
    return out


if __name__ == "__main__":
    print(build(verbose="--verbose" in sys.argv, force="--force" in sys.argv))
