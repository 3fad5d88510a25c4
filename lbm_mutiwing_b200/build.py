"""Builds the CUDA library liblbm_b200.so in-tree with nvcc for sm_100a.

The translation unit holding the FP64 reference-order lattice arithmetic
(plain path, far field) is compiled with -fmad=false so each multiply and add
rounds separately, as the reference's source order prescribes; the immersed
boundary unit spells out its few rounding-sensitive operations with
intrinsics, and the fused FP32 kernel keeps fused multiply-adds.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "liblbm_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
          "--expt-relaxed-constexpr", "-I" + os.path.join(HERE, "..", "include")]
NO_FMA = {"kernels_fp64.cu"}
SOURCES = ["lbm_api.cu", "kernels_fp64.cu", "kernels_fp32.cu", "ibm.cu", "ibm_solver.cu", "err_noalloc.cu"]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(HERE, "..", "include", "lbm_mutiwing.h"))
    objs = []
    for src in SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(BUILD, src.replace(".cu", ".o"))
        objs.append(obj)
        if force or _stale(obj, [path] + headers):
            cmd = [nvcc()] + ARCH + COMMON + (["-fmad=false"] if src in NO_FMA else []) + \
                  ["-Xptxas", "-v"] * verbose + ["-c", path, "-o", obj]
            subprocess.run(cmd, check=True)
    if force or _stale(LIB, objs):
        subprocess.run([nvcc()] + ARCH + ["-shared", "-o", LIB] + objs, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
