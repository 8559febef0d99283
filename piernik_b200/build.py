"""In-tree build of libpiernik_b200.so for sm_100a.

``--fmad=false`` keeps every multiply and add separately rounded, the IEEE
double division and square root are the defaults, and nothing is compiled
with fast-math: this is what makes the kernels reproduce the reference's
gfortran -O2 (SSE2, no FMA) arithmetic bit for bit.  The pk_fast_*.cu units
(the tolerance-mode sweeps) are the exception: they are compiled with
``--fmad=true`` and instantiate only their own kernels.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
PHYS = ["hd1", "hd2", "mhd1", "mhd2", "mhd3"]
# the tolerance-mode units (pk_set_arithmetic(PK_ARITH_FMA)) are the only ones
# compiled with multiply-add contraction
FAST_UNITS = [f"pk_fast_{p}.cu" for p in PHYS]
UNITS = (["pk_api.cu", "pk_noalloc.cu", "pk_peak.cu", "pk_exchange.cpp", "pk_levels.cpp"]
         + [f"pk_phys_{p}.cu" for p in PHYS] + FAST_UNITS)
HEADERS = ["pk_device.cuh", "pk_kernels.cuh", "pk_aux.cuh", "pk_internal.h", "pk_launch.cuh", "pk_adjoint.cuh", "pk_levels.h",
           "pk_adjoint_kernels.cuh", "pk_exchange.h", "pk_fast.cuh"]
DEPS = [os.path.join(CSRC, f) for f in UNITS + HEADERS]
INC = os.path.join(os.path.dirname(HERE), "include")
OUT = os.path.join(HERE, "libpiernik_b200.so")
NVCC = os.environ.get("NVCC", "nvcc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "--fmad=false", "-lineinfo", "-std=c++17",
         "-Xcompiler", "-fPIC,-O2,-ffp-contract=off"]


def needs_build() -> bool:
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    return any(os.path.getmtime(p) > t for p in DEPS + [os.path.join(INC, "piernik_b200.h")])


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile each translation unit to an object (in parallel) and link the .so."""
    if not (force or needs_build()):
        return OUT
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    procs = []
    objs = []
    for unit in UNITS:
        obj = os.path.join(objdir, os.path.splitext(unit)[0] + ".o")
        objs.append(obj)
        flags = [("--fmad=true" if f == "--fmad=false" else f) for f in FLAGS] if unit in FAST_UNITS else FLAGS
        cmd = [NVCC] + flags + (["-Xptxas=-v"] if verbose else []) + ["-I", INC, "-c", "-o", obj,
                                                                    os.path.join(CSRC, unit)]
        procs.append((unit, subprocess.Popen(cmd)))
    bad = [u for u, p in procs if p.wait() != 0]
    if bad:
        raise RuntimeError(f"nvcc failed for {bad}")
    subprocess.check_call([NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", OUT] + objs)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(OUT)
