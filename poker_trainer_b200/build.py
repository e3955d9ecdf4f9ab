"""Builds libdcfr.so in-tree for sm_100a.

nvcc compiles the kernels and the host engine; -fmad=false forbids FMA
contraction and the default IEEE division / denormal handling is kept
(no --use_fast_math), so device arithmetic rounds like the reference's CPU
solver. Every source compiles to its own object under _build/ (in parallel,
only the stale ones), and one nvcc call links them.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libdcfr.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

SOURCES = ["kernels.cu", "terminal.cu", "terminal_fast.cu", "terminal_panel.cu", "terminal_group.cu", "engine.cu", "game.cpp", "capi.cpp",
           "noalloc.cu", "br64.cu", "batch.cu", "mlp.cu", "leaf.cu"]
HEADERS = ["engine.hpp", "game.hpp", "plan.hpp", "warp_terminal.cuh", "row_items.cuh", "batch.hpp", "gemm_tc.cuh",
           "chance_sample.hpp", os.path.join("..", "..", "include", "dcfr.h")]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = [
    *ARCH,
    "-O3", "-lineinfo", "-std=c++17",
    "-fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false",
    "-Xcompiler", "-fPIC,-O3,-ffp-contract=off",
    "-ccbin", "g++",
]
LINK = [*ARCH, "-ccbin", "g++", "--shared", "-cudart", "shared", "-lpthread"]


def _mtime(path: str) -> float:
    return os.path.getmtime(path) if os.path.exists(path) else 0.0


def _headers_mtime() -> float:
    return max([_mtime(os.path.join(CSRC, h)) for h in HEADERS] + [_mtime(os.path.abspath(__file__))])


def _obj(src: str) -> str:
    return os.path.join(OBJ, src + ".o")


def stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return _headers_mtime() > t or any(_mtime(os.path.join(CSRC, s)) > t for s in SOURCES)


def _compile(src: str, verbose: bool) -> None:
    out = _obj(src)
    cmd = [NVCC, *FLAGS, "-c", os.path.join(CSRC, src), "-o", out + ".tmp"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(out + ".tmp", out)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not stale():
        return LIB
    os.makedirs(OBJ, exist_ok=True)
    hdr = _headers_mtime()
    todo = [s for s in SOURCES
            if force or _mtime(_obj(s)) < max(hdr, _mtime(os.path.join(CSRC, s)))]
    workers = max(1, min(len(todo), os.cpu_count() or 1))
    with ThreadPoolExecutor(max_workers=workers) as ex:
        for f in [ex.submit(_compile, s, verbose) for s in todo]:
            f.result()
    cmd = [NVCC, *LINK, *[_obj(s) for s in SOURCES], "-o", LIB + ".tmp"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
