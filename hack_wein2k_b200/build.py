"""Build the in-tree CUDA library liblapw1gpu.so for sm_100a.

    python -m hack_wein2k_b200.build [--force]

nvcc cross-compiles without a GPU; the .so lands next to this file so it
travels with the source tree.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "liblapw1gpu.so")
SOURCES = ["lapw1gpu.cu"]
HEADERS = ["common.cuh", "kernels_fp64.cuh", "split_tc.cuh", "forces.cuh", "sph_tc.cuh"]
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
              "-Xcompiler", "-fPIC", "-shared", "-ccbin", "/usr/bin/g++",
              "-lcublas", "-lcusolver", "-Xlinker", "-rpath", "-Xlinker", "/usr/local/cuda/lib64"]


def _inputs():
    inc = os.path.join(os.path.dirname(HERE), "include", "lapw1gpu.h")
    return [os.path.join(CSRC, f) for f in SOURCES + HEADERS] + [inc]


def stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(f) > t for f in _inputs())


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not stale():
        return LIB
    nvcc = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
    cmd = [nvcc] + NVCC_FLAGS + ["-o", LIB + ".tmp"] + [os.path.join(CSRC, f) for f in SOURCES]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd))
    subprocess.check_call(cmd)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
