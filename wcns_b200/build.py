"""Builds the CUDA library libwcns_b200.so in-tree for sm_100a.

The kernels restate FP64 reference arithmetic operation by operation, so the
library is compiled with -fmad=false (no fused multiply-add contraction);
double division and square root are IEEE round-to-nearest in CUDA.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libwcns_b200.so")
SOURCES = ["capi.cu", "k_rhs_inv.cu", "k_rhs_vis.cu", "k_bc.cu", "k_misc.cu", "k_lhs.cu", "k_metrics.cu", "k_force.cu", "noalloc.cu", "k_sa.cu", "k_sweep_plane.cu", "k_sweep_wide.cu", "k_rhs_mixed.cu", "k_adjoint.cu"]
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-fmad=false", "-std=c++17",
              "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"]

# the mixed-precision residual is not a restatement of the reference's
# operation order, so its file is compiled with multiply-add contraction
CONTRACTED = {"k_rhs_mixed.cu"}


def nvcc():
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(HERE, "..", "include", "wcns_b200.h")]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False, extra=()) -> str:
    if not force and not stale():
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    for src in SOURCES:
        obj = os.path.join(objdir, src.replace(".cu", ".o"))
        flags = [f for f in NVCC_FLAGS if f != "-fmad=false"] if src in CONTRACTED else NVCC_FLAGS
        cmd = [nvcc(), *flags, *extra, "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
        objs.append(obj)
    tmp = LIB + ".tmp"
    subprocess.run([nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", tmp, *objs, "-lcudart"],
                   check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra=["-Xptxas", "-v"] if "--ptxas-v" in sys.argv else [])
