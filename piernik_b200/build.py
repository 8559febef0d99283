"""In-tree build of libpiernik_b200.so for sm_100a.

``--fmad=false`` keeps every multiply and add separately rounded, the IEEE
double division and square root are the defaults, and nothing is compiled
with fast-math: this is what makes the kernels reproduce the reference's
gfortran -O2 (SSE2, no FMA) arithmetic bit for bit.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc", "pk_api.cu")
DEPS = [os.path.join(HERE, "csrc", f) for f in ("pk_api.cu", "pk_device.cuh", "pk_kernels.cuh", "pk_aux.cuh")]
INC = os.path.join(os.path.dirname(HERE), "include")
OUT = os.path.join(HERE, "libpiernik_b200.so")
NVCC = os.environ.get("NVCC", "nvcc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "--fmad=false", "-lineinfo", "-std=c++17",
         "-Xcompiler", "-fPIC,-O2,-ffp-contract=off", "-shared"]


def needs_build() -> bool:
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    return any(os.path.getmtime(p) > t for p in DEPS + [os.path.join(INC, "piernik_b200.h")])


def build(force: bool = False, verbose: bool = False) -> str:
    if force or needs_build():
        cmd = [NVCC] + FLAGS + ["-I", INC, "-o", OUT, SRC]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        subprocess.check_call(cmd)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(OUT)
