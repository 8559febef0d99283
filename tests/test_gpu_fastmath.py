"""The tolerance arithmetic's branch-free reciprocal, quotient and reciprocal
square root (pk_fast.cuh: hardware approximations refined by Newton-Raphson
iterations) against CUDA's correctly rounded operations, in units in the last
place, over operands spanning the magnitudes the sweep meets (1e-30 .. 1e30,
both signs for the quotients)."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "native", "fastmath_harness.cu")
DEPS = [SRC, os.path.join(HERE, "..", "piernik_b200", "csrc", "pk_fast.cuh"),
        os.path.join(HERE, "..", "piernik_b200", "csrc", "pk_device.cuh")]
LIB = os.path.join(HERE, "native", "libfastmath_harness.so")

pytestmark = pytest.mark.gpu


def _lib():
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(p) for p in DEPS):
        subprocess.check_call(["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "--fmad=true",
                               "-std=c++17", "-shared", "-Xcompiler", "-fPIC", "-o", LIB, SRC])
    return C.CDLL(LIB)


def ulps(a, b):
    """|a - b| in units in the last place of b"""
    return np.abs(a - b) / np.spacing(np.abs(b))


def test_newton_refined_ops_within_an_ulp(gpu_lib):
    lib = _lib()
    rng = np.random.default_rng(3)
    n = 1 << 20
    a = rng.standard_normal(n) * 10.0 ** rng.uniform(-30, 30, n)
    b = np.abs(rng.standard_normal(n)) * 10.0 ** rng.uniform(-30, 30, n) + 1e-300
    b[: n // 4] *= -1.0                                   # negative divisors too (not for the roots)
    out = np.empty(8 * n)
    P = C.POINTER(C.c_double)
    rc = lib.fastmath_eval(a.ctypes.data_as(P), b.ctypes.data_as(P), n, out.ctypes.data_as(P))
    assert rc == 0
    o = out.reshape(n, 8)
    pos = b > 0
    assert ulps(o[:, 0], o[:, 1]).max() <= 1.0, "reciprocal"
    assert ulps(o[:, 2], o[:, 3]).max() <= 1.0, "quotient"
    assert ulps(o[pos, 4], o[pos, 5]).max() <= 2.0, "x * rsqrt(x) against sqrt(x)"
    # 1/sqrt(x) is itself rounded twice: within 3 ulp of it is within ~2 of the exact value
    assert ulps(o[pos, 6], o[pos, 7]).max() <= 3.0, "reciprocal square root"
