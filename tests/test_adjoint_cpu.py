"""Vector-Jacobian products of the sweep's building blocks against central
finite differences, on the CPU.

tests/native/adj_harness.cu compiles the same headers the kernels use
(piernik_b200/csrc/pk_device.cuh, pk_adjoint.cuh) for the host.  For random
states covering every branch (supersonic, star and Alfven-fan HLLD states,
B_x = 0, degenerate transverse B, the HLL fallback, moving dust, clipped
floors) the adjoint contracted with a random direction must equal the
directional finite difference of the primal; samples straddling a branch
switch (where two step sizes disagree) are skipped.
"""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "native", "adj_harness.cu")
LIB = os.path.join(HERE, "native", "libadj_harness.so")
dp = C.POINTER(C.c_double)


def P(a):
    return a.ctypes.data_as(dp)


@pytest.fixture(scope="module")
def H():
    deps = [SRC] + [os.path.join(HERE, "..", "piernik_b200", "csrc", f) for f in ("pk_device.cuh", "pk_fast.cuh", "pk_adjoint.cuh")]
    if not os.path.exists(LIB) or any(os.path.getmtime(d) > os.path.getmtime(LIB) for d in deps):
        subprocess.check_call(["nvcc", "-std=c++17", "--fmad=false", "-Xcompiler", "-fPIC,-O2,-ffp-contract=off",
                               "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", LIB, SRC])
    L = C.CDLL(LIB)
    L.h_riemann.argtypes = [C.c_int, dp, dp, C.c_double, C.c_double, dp]
    L.h_riemann_adj.argtypes = [C.c_int, dp, dp, C.c_double, C.c_double, dp, dp, dp]
    L.h_nv.restype = C.c_int
    L.h_slope.restype = C.c_double
    L.h_slope.argtypes = [C.c_int, C.c_double, C.c_double]
    L.h_slope_adj.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double, dp, dp]
    L.h_utoq.argtypes = [C.c_int, dp, C.c_double, dp]
    L.h_utoq_adj.argtypes = [C.c_int, dp, C.c_double, dp, dp]
    L.h_floors.argtypes = [C.c_int, dp, C.c_double, dp, C.POINTER(C.c_uint)]
    L.h_floors_adj.argtypes = [C.c_int, dp, C.c_double, dp, dp]
    return L


def _fd_check(F, ad, h):
    fd = (F(h) - F(-h)) / (2 * h)
    fd2 = (F(h / 4) - F(-h / 4)) / (h / 2)
    if abs(fd - fd2) > 1e-5 * (abs(fd) + 1e-8):
        return None                                     # a branch switch inside the stencil
    return abs(ad - fd) / (abs(fd) + 1e-12)


def _riemann_rel(H, rng, phys, ql, qr, ch=1.3, g=5 / 3):
    nv = H.h_nv(phys)
    fb, vl, vr = rng.standard_normal(nv), rng.standard_normal(nv), rng.standard_normal(nv)
    gl, gr = np.zeros(nv), np.zeros(nv)
    H.h_riemann_adj(phys, P(ql), P(qr), ch, g, P(fb), P(gl), P(gr))

    def F(t):
        f = np.zeros(nv)
        a, b = ql + t * vl, qr + t * vr
        H.h_riemann(phys, P(a), P(b), ch, g, P(f))
        return fb @ f
    return _fd_check(F, gl @ vl + gr @ vr, 1e-6)


def _mhd_pair(rng, case):
    s = rng.uniform
    vx = s(-3, 3) if case == 0 else s(-0.5, 0.5)
    bx = 0.0 if case == 1 else s(-1, 1)
    ql = np.array([s(0.2, 2), vx + s(-.3, .3), s(-1, 1), s(-1, 1), s(0.05, 2), bx, s(-1, 1), s(-1, 1), s(-.1, .1)])
    qr = np.array([s(0.2, 2), vx + s(-.3, .3), s(-1, 1), s(-1, 1), s(0.05, 2), bx * (1.1 if case == 3 else 1.0),
                   s(-1, 1), s(-1, 1), s(-.1, .1)])
    if case == 4:
        ql[6:8] = 0.0
        qr[6:8] = 0.0
    if case == 5:                                       # strong field: HLL fallback of the star B states
        ql[5:8] *= 30.0
        qr[5:8] *= 30.0
    return ql, qr


@pytest.mark.parametrize("case", range(6))
def test_hlld_glm_vjp(H, case):
    rng = np.random.default_rng(10 + case)
    rels = [r for r in (_riemann_rel(H, rng, 1, *_mhd_pair(rng, case)) for _ in range(400)) if r is not None]
    assert len(rels) > 300 and max(rels) < 1e-5


def test_hllc_vjp(H):
    rng = np.random.default_rng(1)
    rels = []
    for t in range(600):
        s = rng.uniform
        vx = s(-3, 3) if t % 3 == 0 else s(-0.5, 0.5)
        ql = np.array([s(0.2, 2), vx + s(-.3, .3), s(-1, 1), s(-1, 1), s(0.05, 2)])
        qr = np.array([s(0.2, 2), vx + s(-.3, .3), s(-1, 1), s(-1, 1), s(0.05, 2)])
        r = _riemann_rel(H, rng, 0, ql, qr, g=1.4)
        if r is not None:
            rels.append(r)
    assert len(rels) > 500 and max(rels) < 1e-5


def test_three_fluid_hlld_vjp(H):
    """Ion (MHD) + neutral (HLLD with B = 0) + dust (gamma < 0) in converging flow."""
    rng = np.random.default_rng(2)
    rels = []
    for _ in range(300):
        s = rng.uniform
        mk = lambda: np.concatenate([[s(.2, 2), s(-.5, .5), s(-1, 1), s(-1, 1), s(.05, 2)],
                                     [s(.2, 2), s(-.5, .5), s(-1, 1), s(-1, 1), s(.05, 2)],
                                     [s(.2, 2), s(-.5, .5), s(-1, 1), s(-1, 1)],
                                     [s(-1, 1), s(-1, 1), s(-1, 1), s(-.1, .1)]])
        ql, qr = mk(), mk()
        ql[14] = qr[14] = s(-1, 1)
        if ql[11] < qr[11]:
            ql[11], qr[11] = qr[11], ql[11]
        r = _riemann_rel(H, rng, 2, ql, qr)
        if r is not None:
            rels.append(r)
    assert len(rels) > 250 and max(rels) < 1e-5


@pytest.mark.parametrize("lim", range(4))
def test_limiter_vjp(H, lim):
    rng = np.random.default_rng(3 + lim)
    rels = []
    for t in range(1000):
        dl, dr = rng.standard_normal(2)
        if t % 3 == 0:
            dr = dl * rng.uniform(0.1, 3)
        sb = rng.standard_normal()
        a, b = C.c_double(), C.c_double()
        H.h_slope_adj(lim, dl, dr, sb, C.byref(a), C.byref(b))
        vl, vr = rng.standard_normal(2)
        r = _fd_check(lambda t: sb * H.h_slope(lim, dl + t * vl, dr + t * vr), a.value * vl + b.value * vr, 1e-7)
        if r is not None:
            rels.append(r)
    assert len(rels) > 900 and max(rels) < 1e-5


def _cell(rng, phys, nv):
    u = rng.uniform(0.3, 2, nv)
    u[1:4] = rng.uniform(-1, 1, 3)
    if phys >= 1:
        u[nv - 4:nv] = rng.uniform(-1, 1, 4)
    if phys == 2:
        u[6:9] = rng.uniform(-1, 1, 3)
        u[11:14] = rng.uniform(-1, 1, 3)
    return u


@pytest.mark.parametrize("phys,nv", [(0, 5), (1, 9), (2, 18)])
def test_utoq_vjp(H, phys, nv):
    rng = np.random.default_rng(20 + phys)
    for _ in range(300):
        u = _cell(rng, phys, nv)
        u[4] = 3.0
        qb, v, ub = rng.standard_normal(nv), rng.standard_normal(nv), np.zeros(nv)
        H.h_utoq_adj(phys, P(u), 5 / 3, P(qb), P(ub))

        def F(t):
            q = np.zeros(nv)
            x = u + t * v
            H.h_utoq(phys, P(x), 5 / 3, P(q))
            return qb @ q
        r = _fd_check(F, ub @ v, 1e-6)
        assert r is not None and r < 1e-6


@pytest.mark.parametrize("phys,nv", [(0, 5), (1, 9), (2, 18)])
def test_floors_vjp(H, phys, nv):
    """internal_sources + care_for_positives, with the density and
    internal-energy floors clipping in a large share of the samples."""
    rng = np.random.default_rng(30 + phys)
    rels, clipped = [], 0
    for t in range(400):
        u = _cell(rng, phys, nv)
        kin = 0.5 * (u[1:4] ** 2).sum() / u[0]
        mag = 0.5 * (u[nv - 4:nv - 1] ** 2).sum() if phys >= 1 else 0.0
        u[4] = kin + mag + rng.uniform(-0.2, 0.5)
        if t % 5 == 0:
            u[0] = rng.uniform(-0.01, 0.002)
        lb, v, out = rng.standard_normal(nv), rng.standard_normal(nv), np.zeros(nv)
        rec = (C.c_uint * 2)()
        H.h_floors(phys, P(u), 5 / 3, P(np.zeros(nv)), rec)
        clipped += rec[1] != 0 or rec[0] != 0
        H.h_floors_adj(phys, P(u), 5 / 3, P(lb), P(out))

        def F(t):
            q = np.zeros(nv)
            x = u + t * v
            H.h_floors(phys, P(x), 5 / 3, P(q), (C.c_uint * 2)())
            return lb @ q
        r = _fd_check(F, out @ v, 1e-8)
        if r is not None:
            rels.append(r)
    assert clipped > 100 and len(rels) > 350 and max(rels) < 1e-5
