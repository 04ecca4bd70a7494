"""Build libeddy_b200.so (all CUDA kernels + the C ABI) in-tree for sm_100a.

Usage: python -m eddy_hybrid_b200.build   (or eddy_hybrid_b200.build.build())
The plain FP64 kernels are compiled with -fmad=false so their rounding follows
the reference's operation order; nvcc cross-compiles without a GPU.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libeddy_b200.so")
OBJ = os.path.join(HERE, "_build")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

# per-translation-unit flags: exact-order FP64 kernels get -fmad=false
UNITS = {
    "eddy_ctx.cu": ["-fmad=false"],
    "k_momentum.cu": ["-fmad=false"],
    "k_poisson.cu": ["-fmad=false"],
    "k_density.cu": ["-fmad=false"],
    "k_sgs.cu": ["-fmad=false"],
    "k_sgs32.cu": [],
    "k_noalloc.cu": ["-fmad=false"],
    "k_selftest.cu": [],
    "k_mlp.cu": [],
    "k_mixed.cu": [],
    "k_xform.cu": [],
    "k_xform64.cu": [],
    "k_ib.cu": ["-fmad=false"],
    "k_implicit.cu": ["-fmad=false"],
    "k_diag.cu": ["-fmad=false"],
    "k_force.cu": ["-fmad=false"],
    "host_eigen.cpp": [],
    "host_restart.cpp": [],
}


def _newer(src_list, out):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(s) > t for s in src_list)


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    hdrs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hdrs.append(os.path.join(HERE, "..", "include", "eddy_b200.h"))
    objs = []
    for unit, extra in UNITS.items():
        src = os.path.join(CSRC, unit)
        obj = os.path.join(OBJ, unit + ".o")
        objs.append(obj)
        if not force and not _newer([src] + hdrs, obj):
            continue
        cmd = [NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
               "-I", os.path.join(HERE, "..", "include"), *extra, "-c", src, "-o", obj]
        if unit.endswith(".cpp"):
            cmd = [NVCC, *ARCH, "-O2", "-std=c++17", "-Xcompiler", "-fPIC,-ffp-contract=off",
                   "-I", os.path.join(HERE, "..", "include"), "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    if force or _newer(objs, OUT):
        cmd = [NVCC, *ARCH, "-shared", "-cudart", "static", "-o", OUT, *objs]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
