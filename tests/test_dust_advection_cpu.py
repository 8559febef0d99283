"""The pressureless dust fluid of the split sweep (dust_cs = 0, HLLC with
gamma < 0: riemann_hlld_u's dust branch) on an exact solution, on the CPU:
a smooth density pulse moving at uniform velocity 1 once around a periodic
unit box comes back to its initial profile.  The L1 error must fall at
second order (measured 14.5-fold (van Leer) and 13.8-fold (moncen) from 64
to 256 cells, to 0.00044 / 0.00038) and the mass must stay constant to
rounding.  The reference holds no known answer for the dust fluid."""
import numpy as np
import pytest

import oracle
from piernik_b200.config import Setup


def advect(n, lim):
    s = Setup(n=(n, 1, 1), fluids=[("dst", -1.0)], magnetic=False, limiter=lim, limiter_b=lim,
              xmin=(0.0, 0.0, 0.0), xmax=(1.0, 1.0, 1.0), cfl=0.7, tend=1.0)
    g, ext = s.guards, s.ext
    x = (np.arange(ext[0]) - g[0] + 0.5) / n
    rho = 1.0 + 0.5 * np.sin(2.0 * np.pi * x)
    u = np.zeros((ext[2], ext[1], ext[0], s.nvar))
    u[..., 0] = rho
    u[..., 1] = rho * 1.0
    ob = oracle.OracleBlock(s, u)
    ob.fill_guards()
    for _ in range(100000):
        if ob.state.t >= 1.0 * (1.0 - 1e-12):
            break
        assert ob.run(1) == 0
    assert abs(ob.state.t - 1.0) <= 1e-12
    inner = slice(g[0], g[0] + n)
    got = ob.u[0, 0, inner, 0]
    return float(np.mean(np.abs(got - rho[inner]))), float(abs(got.sum() / n - 1.0))


@pytest.mark.parametrize("lim", ["vanleer", "moncen"])
def test_dust_pulse_returns(lim):
    e64, m64 = advect(64, lim)
    e256, m256 = advect(256, lim)
    assert e256 < 6e-4, (lim, e64, e256)
    assert e64 / e256 > 12.0, (lim, e64, e256)
    assert m64 < 1e-14 and m256 < 1e-14
