"""Build the in-tree CUDA library libawsem_gpu.so for sm_100a.

The library is plain nvcc output (no torch extension machinery): C++ host
code for the model and the C ABI, CUDA kernels for Blackwell (sm_100a).
Built artefacts stay inside the package directory so they travel with the
source tree.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
LIB = os.path.join(HERE, "libawsem_gpu.so")
BUILD = os.path.join(HERE, "_build")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# -fmad=false: no multiply-add contraction left to the compiler.  Every
# product and sum is then rounded on its own, in source order, as the x86-64
# CPU build of the reference computes them, and identically in every kernel
# that inlines the same device code (the per-pass kernels and the persistent
# step kernel give bit-identical trajectories).  Fused operations are written
# out where they are wanted (__fmaf_rn / __fma_rn).
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-fmad=false", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
              "--expt-relaxed-constexpr", "-I" + CSRC, "-I" + INCLUDE]
SOURCES = ["awsem_model.cpp", "awsem_engine.cu", "awsem_noalloc.cu"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(INCLUDE, "awsem_gpu.h"))
    headers.append(os.path.abspath(__file__))  # the flags above
    objs = []
    for src in SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(BUILD, src + ".o")
        objs.append(obj)
        if force or _stale(obj, [path] + headers):
            cmd = [nvcc()] + ARCH + NVCC_FLAGS + ["-c", path, "-o", obj]
            if src.endswith(".cpp"):
                cmd = [nvcc()] + ARCH + NVCC_FLAGS + ["-x", "cu", "-c", path, "-o", obj]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
    if force or _stale(LIB, objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
