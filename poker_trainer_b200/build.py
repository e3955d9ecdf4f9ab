"""Builds libdcfr.so in-tree for sm_100a.

nvcc compiles the kernels and the host engine; -fmad=false forbids FMA
contraction and the default IEEE division / denormal handling is kept
(no --use_fast_math), so device arithmetic rounds like the reference's CPU
solver.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libdcfr.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

SOURCES = ["kernels.cu", "terminal.cu", "terminal_fast.cu", "engine.cu", "game.cpp", "capi.cpp", "noalloc.cu", "br64.cu", "batch.cu", "mlp.cu", "leaf.cu"]
HEADERS = ["engine.hpp", "game.hpp", "plan.hpp", "warp_terminal.cuh", "row_items.cuh", "batch.hpp", "gemm_tc.cuh", os.path.join("..", "..", "include", "dcfr.h")]

FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false",
    "-Xcompiler", "-fPIC,-O3,-ffp-contract=off",
    "-ccbin", "g++",
    "--shared", "-cudart", "shared",
]


def stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    for f in SOURCES + HEADERS + [os.path.basename(__file__)]:
        path = os.path.join(CSRC, f) if f != os.path.basename(__file__) else os.path.abspath(__file__)
        if os.path.exists(path) and os.path.getmtime(path) > t:
            return True
    return False


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not stale():
        return LIB
    cmd = [NVCC, *FLAGS, *[os.path.join(CSRC, s) for s in SOURCES], "-o", LIB + ".tmp"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
