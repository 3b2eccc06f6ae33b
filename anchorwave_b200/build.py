"""Builds libaw_b200.so (all CUDA kernels + the C ABI) in-tree for sm_100a.

The shared library is the product: Python (anchorwave_b200.*), C/C++ callers
(include/anchorwave_b200.h) and bench.py all reach the kernels through it.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libaw_b200.so")
SOURCES = ["ksw2_full.cu", "ksw2_band.cu", "ksw2_exact.cu", "ksw2_api.cu", "ksw2_noalloc.cu", "wfa.cu", "wfa_api.cu",
           "wfa2_compat.cu", "serve.cu", "peak.cu", "rows.cu", "rescue.cu", "summary.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def sources():
    return [os.path.join(CSRC, s) for s in SOURCES if os.path.exists(os.path.join(CSRC, s))]


def build(verbose: bool = False, ptxas_info: bool = False, force: bool = False) -> str:
    srcs = sources()
    deps = srcs + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    deps.append(os.path.join(ROOT, "include", "anchorwave_b200.h"))
    if not force and os.path.exists(LIB) and all(os.path.getmtime(LIB) >= os.path.getmtime(d) for d in deps):
        return LIB
    cmd = [nvcc(), *ARCH, "-lineinfo", "-O3", "-std=c++17", "--expt-relaxed-constexpr",
           "-Xcompiler", "-fPIC,-O2", "-shared", "-o", LIB, *srcs, "-ldl", "-lpthread"]
    if ptxas_info:
        cmd.insert(1, "-Xptxas=-v")
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose=True, ptxas_info="-v" in sys.argv, force="-f" in sys.argv)
