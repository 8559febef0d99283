"""The oracle's split scheme against the exact solution of the Euler
Riemann problem (Sod's shock tube), on the CPU.

The reference holds known answers for this path only for the circularly
polarised Alfven wave (CPAW, tests/test_cpaw.py), which exercises the unsplit
scheme with the van Leer limiter.  This test pins the other pieces of the
split sweep against physics rather than reference data: HLLC
(riemann_hlld_u) with each limiter (van Leer, minmod, moncen, superbee) must
converge to the exact solution -- density L1 error below a bound at 400
cells (measured 0.0012-0.0024) and falling at least 2.8-fold from 100 to 400
cells (measured 3.2-3.6: first order at the discontinuities) -- and the
shock and the rarefaction head must sit where the exact solution puts them.

The exact solution follows the published method of E. F. Toro, Riemann
Solvers and Numerical Methods for Fluid Dynamics (3rd ed., Springer 2009),
ch. 4: the star pressure from Newton iterations on the pressure function,
then sampling along x/t.
"""
import math

import numpy as np
import pytest

import oracle
from piernik_b200.config import BND_OUT, Setup

GAMMA = 1.4
LEFT, RIGHT = (1.0, 0.0, 1.0), (0.125, 0.0, 0.1)      # (rho, u, p): Sod (1978)
TEND, X0 = 0.2, 0.5


def _pressure_function(p, rho, pk, ck, g):
    if p > pk:                                          # shock (Toro eq. 4.21)
        a, b = 2.0 / ((g + 1.0) * rho), (g - 1.0) / (g + 1.0) * pk
        f = (p - pk) * math.sqrt(a / (p + b))
        df = math.sqrt(a / (b + p)) * (1.0 - (p - pk) / (2.0 * (b + p)))
    else:                                               # rarefaction (eq. 4.26)
        f = 2.0 * ck / (g - 1.0) * ((p / pk) ** ((g - 1.0) / (2.0 * g)) - 1.0)
        df = 1.0 / (rho * ck) * (p / pk) ** (-(g + 1.0) / (2.0 * g))
    return f, df


def exact_riemann(left, right, g, xi):
    """(rho, u, p) of the exact Riemann solution at similarity coordinates xi = (x - x0) / t."""
    rl, ul, pl = left
    rr, ur, pr = right
    cl, cr = math.sqrt(g * pl / rl), math.sqrt(g * pr / rr)
    p = max(1e-10, 0.5 * (pl + pr))
    for _ in range(100):                                # Newton on f_L + f_R + du = 0 (eq. 4.5)
        fl, dfl = _pressure_function(p, rl, pl, cl, g)
        fr, dfr = _pressure_function(p, rr, pr, cr, g)
        pn = max(1e-10, p - (fl + fr + ur - ul) / (dfl + dfr))
        if abs(pn - p) < 1e-14 * (pn + p):
            p = pn
            break
        p = pn
    fl, _ = _pressure_function(p, rl, pl, cl, g)
    fr, _ = _pressure_function(p, rr, pr, cr, g)
    us = 0.5 * (ul + ur) + 0.5 * (fr - fl)
    gm, gp = (g - 1.0) / (g + 1.0), (g - 1.0) / (2.0 * g)
    out = np.empty((len(xi), 3))
    for i, s in enumerate(xi):                          # sampling (section 4.5)
        if s <= us:                                     # left of the contact
            if p > pl:
                sl = ul - cl * math.sqrt((g + 1.0) / (2.0 * g) * p / pl + gp)
                out[i] = (rl, ul, pl) if s <= sl else (rl * (p / pl + gm) / (gm * p / pl + 1.0), us, p)
            else:
                shl, stl = ul - cl, us - cl * (p / pl) ** gp
                if s <= shl:
                    out[i] = (rl, ul, pl)
                elif s >= stl:
                    out[i] = (rl * (p / pl) ** (1.0 / g), us, p)
                else:
                    c = 2.0 / (g + 1.0) * (cl + (g - 1.0) / 2.0 * (ul - s))
                    out[i] = (rl * (c / cl) ** (2.0 / (g - 1.0)), 2.0 / (g + 1.0) * (cl + (g - 1.0) / 2.0 * ul + s),
                              pl * (c / cl) ** (2.0 * g / (g - 1.0)))
        else:                                           # right of the contact
            if p > pr:
                sr = ur + cr * math.sqrt((g + 1.0) / (2.0 * g) * p / pr + gp)
                out[i] = (rr, ur, pr) if s >= sr else (rr * (p / pr + gm) / (gm * p / pr + 1.0), us, p)
            else:
                shr, stp = ur + cr, us + cr * (p / pr) ** gp
                if s >= shr:
                    out[i] = (rr, ur, pr)
                elif s <= stp:
                    out[i] = (rr * (p / pr) ** (1.0 / g), us, p)
                else:
                    c = 2.0 / (g + 1.0) * (cr - (g - 1.0) / 2.0 * (ur - s))
                    out[i] = (rr * (c / cr) ** (2.0 / (g - 1.0)), 2.0 / (g + 1.0) * (-cr + (g - 1.0) / 2.0 * ur + s),
                              pr * (c / cr) ** (2.0 * g / (g - 1.0)))
    return out, p, us


def sod(n, lim):
    """Density at the cell centres after the oracle ran Sod's tube to TEND."""
    s = Setup(n=(n, 1, 1), fluids=[("neu", GAMMA)], magnetic=False, limiter=lim, limiter_b=lim,
              xmin=(0.0, 0.0, 0.0), xmax=(1.0, 1.0, 1.0), bnd=((BND_OUT, BND_OUT),) * 3, cfl=0.7, tend=TEND)
    ext = s.ext
    g = s.guards
    u = np.zeros((ext[2], ext[1], ext[0], s.nvar))
    x = s.xmin[0] + (np.arange(ext[0]) - g[0] + 0.5) * s.dl[0]
    left = x < X0
    rho = np.where(left, LEFT[0], RIGHT[0])
    p = np.where(left, LEFT[2], RIGHT[2])
    u[..., 0] = rho
    u[..., 4] = p / (GAMMA - 1.0)
    ob = oracle.OracleBlock(s, u)
    ob.fill_guards()
    for _ in range(20000):
        if ob.state.t >= TEND * (1.0 - 1e-12):
            break
        assert ob.run(1) == 0
    assert abs(ob.state.t - TEND) <= 1e-9
    xc = x[g[0]:g[0] + n]
    return xc, ob.u[0, 0, g[0]:g[0] + n, 0]


@pytest.mark.parametrize("lim,bound", [("vanleer", 0.003), ("minmod", 0.004), ("moncen", 0.003),
                                       ("superbee", 0.003)])
def test_sod_converges_to_exact_solution(lim, bound):
    errs = {}
    for n in (100, 400):
        xc, rho = sod(n, lim)
        exact, _, _ = exact_riemann(LEFT, RIGHT, GAMMA, (xc - X0) / TEND)
        errs[n] = float(np.mean(np.abs(rho - exact[:, 0])))
    assert errs[400] < bound, (lim, errs)
    assert errs[100] / errs[400] > 2.8, (lim, errs)


def test_sod_wave_positions():
    """Shock, contact and rarefaction head where the exact solution has them
    (within two cells at 400 cells, moncen)."""
    n = 400
    xc, rho = sod(n, "moncen")
    exact, ps, us = exact_riemann(LEFT, RIGHT, GAMMA, (xc - X0) / TEND)
    dx = 1.0 / n
    # the shock: the last cell above the mid-value between the post-shock and right densities
    post = exact[np.argmin(np.abs(xc - (X0 + us * TEND + 0.05))), 0]
    mid = 0.5 * (post + RIGHT[0])
    shock_num = xc[np.nonzero(rho > mid)[0].max()]
    shock_ex = xc[np.nonzero(exact[:, 0] > mid)[0].max()]
    assert abs(shock_num - shock_ex) <= 2 * dx
    # the rarefaction head: the first cell where the density drops below the left state
    head_num = xc[np.nonzero(rho < LEFT[0] - 1e-3)[0].min()]
    head_ex = X0 - math.sqrt(GAMMA * LEFT[2] / LEFT[0]) * TEND
    assert abs(head_num - head_ex) <= 3 * dx
    assert 0.25 < ps < 0.35                             # p* of Sod's problem: 0.30313 (Toro table 4.2)
