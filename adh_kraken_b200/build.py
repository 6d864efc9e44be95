"""Build the in-tree CUDA library libadh_sw2_gpu.so for sm_100a.

The element kernels (sw2_kernels.cu) are compiled with --fmad=false so their
results are bit-identical to the reference CPU build; the linear-algebra kernels
keep FMA contraction.  Host code is compiled without floating-point contraction
(the element geometry it computes must match the reference's selem2d/selem1d).
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libadh_sw2_gpu.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-ffp-contract=off", "--expt-relaxed-constexpr",
          "-I" + os.path.join(HERE, "..", "include")]
# (source, extra flags)
UNITS = [
    ("sw2_kernels.cu", ["--fmad=false"]),
    ("la_kernels.cu", []),
    ("ilu_kernels.cu", []),
    ("amg_kernels.cu", []),
    ("gmres_kernels.cu", []),
    ("gnn_kernels.cu", []),
    ("sw2_capi.cu", []),
]


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(LIBDIR, exist_ok=True)
    objdir = os.path.join(LIBDIR, "obj")
    os.makedirs(objdir, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(HERE, "..", "include", "adh_sw2_gpu.h"))
    objs = []
    for src, extra in UNITS:
        s = os.path.join(CSRC, src)
        o = os.path.join(objdir, src.replace(".cu", ".o"))
        objs.append(o)
        if force or _stale(o, [s, *headers, __file__]):
            cmd = [NVCC, *ARCH, *COMMON, *extra, "-c", s, "-o", o]
            if verbose:
                print(" ".join(cmd), file=sys.stderr)
            subprocess.run(cmd, check=True)
    if force or _stale(LIB, objs):
        cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(verbose=True, force="--force" in sys.argv))
