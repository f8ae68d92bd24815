"""Builds the CUDA library in-tree: saddlepoint_b200/_build/libsaddlepoint_b200.so (sm_100a).

    python -m saddlepoint_b200.build [--force]

Every translation unit is compiled for sm_100a with --fmad=false (each multiply
and add rounded separately, as the reference's Rust code computes them) and
linked into one shared library exporting the C ABI of include/saddlepoint_b200.h.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_build")
LIB = os.path.join(OUT, "libsaddlepoint_b200.so")
NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-std=c++17", "-O3", "-lineinfo", "--fmad=false", "-Xcompiler", "-fPIC,-O3", "-Xptxas", "-O3"]
CU = ["backend.cu", "solver.cu", "batch.cu", "serve.cu", "noalloc.cu", "triplets.cu"]
CPP = ["host.cpp", "mps.cpp", "presolve.cpp", "polish.cpp"]
HEADERS = ["common.cuh", "internal.cuh", "tiles.cuh", "stream.cuh", "sell.cuh", "control.cuh", "solver_kernels.cuh", "solver_state.h", "batch_kernels.cuh"]


def _sources():
    return [f for f in CU + CPP if os.path.exists(os.path.join(CSRC, f))]


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in _sources() + HEADERS if os.path.exists(os.path.join(CSRC, f))]
    deps.append(os.path.join(HERE, "..", "include", "saddlepoint_b200.h"))
    deps.append(os.path.abspath(__file__))
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src: str) -> str:
    obj = os.path.join(OUT, src + ".o")
    cmd = [NVCC, *ARCH, *FLAGS, "-c", os.path.join(CSRC, src), "-o", obj]
    subprocess.run(cmd, check=True)
    return obj


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return LIB
    os.makedirs(OUT, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=max(1, min(8, os.cpu_count() or 1))) as ex:
        objs = list(ex.map(_compile, _sources()))
    cmd = [NVCC, *ARCH, "-shared", "-o", LIB + ".tmp", *objs, "-lcudart", "-lpthread"]
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    if verbose:
        print(LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
