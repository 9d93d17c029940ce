"""Build the sm_100a shared library in-tree (nvcc cross-compiles; no GPU)."""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libcublox_b200.so")
SOURCES = ["csrc/kernels.cu", "csrc/raycast_binned.cu", "csrc/raycast_split.cu", "csrc/capi.cu",
           "csrc/noalloc.cu", "csrc/batch.cu", "csrc/server.cpp", "csrc/probe.cu"]
HEADERS = ["csrc/kernels.cuh", "csrc/exact_fp.cuh", "csrc/ray_walk.cuh", "csrc/fold.cuh", "csrc/far_walk.cuh", "csrc/dda_jump.cuh", "csrc/grid_internal.hpp", "../include/cublox_b200.h"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    # Every FP32 operation of the path is spelled with an explicit rounding
    # intrinsic; nothing may be fused implicitly.
    "-fmad=false",
    "-shared", "-Xcompiler", "-fPIC,-ffp-contract=off,-O2,-pthread",
]


def _stale(out: str, inputs: list[str]) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(os.path.join(HERE, p)) > t for p in inputs)


def build(force: bool = False, verbose: bool = False, extra: list[str] | None = None) -> str:
    if force or _stale(LIB, SOURCES + HEADERS):
        cmd = ["nvcc", *NVCC_FLAGS, *(extra or []), "-o", LIB, *SOURCES]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.check_call(cmd, cwd=HERE)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra=["-Xptxas", "-v"] if "--ptxas" in sys.argv else None)
