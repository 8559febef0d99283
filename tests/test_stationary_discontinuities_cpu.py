"""Exact properties of the split sweep's Riemann solvers, on the CPU.

HLLC (Toro, Spruce & Speares 1994) resolves an isolated stationary contact
exactly, and HLLD (Miyoshi & Kusano 2005) an isolated stationary contact
(B_x != 0, continuous transverse field) and a stationary tangential
discontinuity (B_x = 0, transverse field jumping with the total pressure
balanced).  With moncen reconstruction and outflow boundaries every value of
such a state stays bit for bit what it was over 40 steps: this pins the
star-state branches of riemann_hlld_u and riemann_hlld (the degenerate
speed test, the contact speed sm = 0, the B_x = 0 branch) against the
solvers' published design rather than reference data."""
import numpy as np
import pytest

import oracle
from piernik_b200.config import BND_OUT, Setup


def _run(mag, kind, nsteps=40, n=64):
    gam = 5.0 / 3.0 if mag else 1.4
    s = Setup(n=(n, 1, 1), fluids=[("ion", gam)] if mag else [("neu", gam)], magnetic=mag, limiter="moncen",
              limiter_b="moncen", xmin=(0.0, 0.0, 0.0), xmax=(1.0, 1.0, 1.0), bnd=((BND_OUT, BND_OUT),) * 3, cfl=0.7)
    g, ext = s.guards, s.ext
    x = (np.arange(ext[0]) - g[0] + 0.5) / n
    left = x < 0.5
    u = np.zeros((ext[2], ext[1], ext[0], s.nvar))
    rho = np.where(left, 1.0, 0.3)
    p = np.full_like(x, 1.0)
    b = psi = None
    pm = 0.0
    if mag:
        b = np.zeros((ext[2], ext[1], ext[0], 3))
        psi = np.zeros((ext[2], ext[1], ext[0]))
        if kind == "contact":
            b[..., 0], b[..., 1], b[..., 2] = 0.7, 0.4, -0.2
        else:
            by = np.where(left, 0.8, 0.3)
            b[..., 1] = by
            p = 1.0 + 0.5 * (0.8 ** 2 - by ** 2)
        pm = 0.5 * (b[..., 0] ** 2 + b[..., 1] ** 2 + b[..., 2] ** 2)
    u[..., 0] = rho
    u[..., 4] = p / (gam - 1.0) + pm
    ob = oracle.OracleBlock(s, u, b, psi)
    ob.fill_guards()
    u0 = ob.u.copy()
    b0 = ob.b.copy() if mag else None
    for _ in range(nsteps):
        assert ob.run(1) == 0
    assert ob.state.t > 0.25
    return ob, u0, b0


@pytest.mark.parametrize("mag,kind", [(False, "contact"), (True, "contact"), (True, "tangential")])
def test_stationary_discontinuity_is_exact(mag, kind):
    ob, u0, b0 = _run(mag, kind)
    assert np.array_equal(ob.u, u0)
    if mag:
        assert np.array_equal(ob.b, b0)
