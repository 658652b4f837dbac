"""Builds the CUDA library in-tree (sm_100a).

``python -m andfn_b200.build`` compiles ``csrc/*.cu`` and ``csrc/*.cpp`` with
nvcc into ``andfn_b200/libandfn_b200.so``.  No GPU is needed to build.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libandfn_b200.so")
SOURCES = [os.path.join(HERE, "csrc", f) for f in ("solver.cu", "geometry.cu", "sparse_lu.cpp")]
DEPS = SOURCES + [os.path.join(HERE, "csrc", f) for f in ("dmath.cuh", "sparse_lu.h", "track.cuh")] + [
    os.path.join(os.path.dirname(HERE), "include", "andfn_b200.h")]
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
              "-Xcompiler", "-fPIC,-O3,-fopenmp", "-shared", "-diag-suppress", "550", "-lgomp"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return "nvcc"


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(d) > t for d in DEPS if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not needs_build():
        return LIB
    cmd = [nvcc()] + NVCC_FLAGS + ["-o", LIB] + SOURCES
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
