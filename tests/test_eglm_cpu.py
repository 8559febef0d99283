"""The E-GLM sources of the oracle (hdc.F90:355-457, ``use_eglm``) on the
CPU: the identity where div B and grad psi vanish, and bit-equal to an
independent NumPy restatement of the reference's statements on a noisy
periodic block (divB of order 2 and grad psi from the +-1 neighbours, then
per cell m, B, E and psi in the reference's order, dot products accumulated
from zero).  The reference holds no test or golden data for E-GLM, so this
pins the restatement's arithmetic, not its agreement with a reference run."""
import numpy as np

import oracle
from helpers import random_state, setup_for


def _numpy_eglm(s, u, b, psi, dt):
    g = s.guards
    n = s.n
    D = [1 if n[d] > 1 else 0 for d in range(3)]
    sl = tuple(slice(g[d], g[d] + n[d]) for d in (2, 1, 0))

    def shift(a, d, k):                                   # a at cell +k along d (array axes z, y, x)
        ax = 2 - d
        idx = [slice(g[e], g[e] + n[e]) for e in (2, 1, 0)]
        idx[ax] = slice(g[d] + k * D[d], g[d] + n[d] + k * D[d])
        return a[tuple(idx)]

    t = [(shift(b[..., d], d, 1) - shift(b[..., d], d, -1)) / s.dl[d] for d in range(3)]
    q = 0.5 * ((t[0] + t[1]) + t[2])
    gp = [(0.5 * (shift(psi, d, 1) - shift(psi, d, -1))) / s.dl[d] for d in range(3)]
    uu, bb, pp = u.copy(), b.copy(), psi.copy()
    rho = uu[sl + (0,)]
    m = [uu[sl + (1 + c,)] - (dt * q) * bb[sl + (c,)] for c in range(3)]
    v = [m[c] / rho for c in range(3)]
    B = [bb[sl + (c,)] - (dt * q) * v[c] for c in range(3)]
    vb = ((0.0 + v[0] * B[0]) + v[1] * B[1]) + v[2] * B[2]
    bg = ((0.0 + B[0] * gp[0]) + B[1] * gp[1]) + B[2] * gp[2]
    vg = ((0.0 + v[0] * gp[0]) + v[1] * gp[1]) + v[2] * gp[2]
    for c in range(3):
        uu[sl + (1 + c,)] = m[c]
        bb[sl + (c,)] = B[c]
    uu[sl + (4,)] = uu[sl + (4,)] - dt * (q * vb - bg)
    pp[sl] = pp[sl] - dt * vg
    return uu, bb, pp


def test_eglm_identity_without_sources():
    s = setup_for("mhd", n=(10, 8, 6), lim="vanleer").replace(use_eglm=True)
    u, b, psi = random_state(s, seed=3)
    b[...] = np.array([0.3, -0.2, 0.1])
    psi[...] = 0.7
    ob = oracle.OracleBlock(s, u, b, psi)
    ob.fill_guards()
    u0, b0, p0 = ob.u.copy(), ob.b.copy(), ob.psi.copy()
    ob.eglm(0.01)
    assert np.array_equal(ob.u, u0) and np.array_equal(ob.b, b0) and np.array_equal(ob.psi, p0)


def test_eglm_off_is_a_no_op():
    s = setup_for("mhd", n=(10, 8, 6), lim="vanleer")
    ob = oracle.OracleBlock(s, *random_state(s, seed=4))
    ob.fill_guards()
    u0 = ob.u.copy()
    ob.eglm(0.01)
    assert np.array_equal(ob.u, u0)


def test_eglm_equals_numpy_restatement():
    for n in [(12, 10, 8), (16, 12, 1)]:
        s = setup_for("mhd", n=n, lim="vanleer").replace(use_eglm=True)
        ob = oracle.OracleBlock(s, *random_state(s, seed=5))
        ob.fill_guards()
        want_u, want_b, want_p = _numpy_eglm(s, ob.u, ob.b, ob.psi, 0.013)
        ob.eglm(0.013)
        g = s.guards
        sl = tuple(slice(g[d], g[d] + s.n[d]) for d in (2, 1, 0))
        assert np.array_equal(ob.u[sl], want_u[sl]), n
        assert np.array_equal(ob.b[sl], want_b[sl]), n
        assert np.array_equal(ob.psi[sl], want_p[sl]), n
