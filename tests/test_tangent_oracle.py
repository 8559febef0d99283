"""The tangent-linear oracle (oracle/pk_tangent.cpp): its value part is the
oracle bit for bit, and its derivative part is the directional derivative
of the oracle's fixed-dt map, checked against central differences where
those are well defined (one-cell seeds on a smooth state)."""
import numpy as np
import pytest

import oracle
import tangent
from helpers import setup_for, smooth_state


@pytest.mark.parametrize("phys,lim", [("hd", "vanleer"), ("mhd", "moncen")])
def test_tangent_values_are_the_oracle(oracle_lib, phys, lim):
    s = setup_for(phys, n=(10, 8, 6), lim=lim)
    u, b, psi = smooth_state(s, seed=3)
    dts = [0.01, 0.012]
    ob = oracle.OracleBlock(s, u, b, psi)
    ob.fill_guards()
    assert ob.run_fixed(dts) == 0
    ob.fill_guards()
    rng = np.random.default_rng(0)
    du = rng.standard_normal(u.shape)
    db = rng.standard_normal(b.shape) if b is not None else None
    dp = rng.standard_normal(psi.shape) if psi is not None else None
    (tu, tb, tp), _ = tangent.jvp(s, u, b, psi, du, db, dp, dts)
    assert np.array_equal(tu.view(np.uint64), ob.u.view(np.uint64))
    if s.magnetic:
        assert np.array_equal(tb.view(np.uint64), ob.b.view(np.uint64))
        assert np.array_equal(tp.view(np.uint64), ob.psi.view(np.uint64))


@pytest.mark.parametrize("phys", ["hd", "mhd"])
def test_tangent_matches_central_differences(oracle_lib, phys):
    s = setup_for(phys, n=(10, 8, 6), lim="vanleer")
    u, b, psi = smooth_state(s, seed=4)
    dts = [0.01, 0.012]
    g = s.guards
    rng = np.random.default_rng(5)
    worst = 0.0
    for trial in range(4):
        k, j, i = (g[2] + rng.integers(0, s.n[2]), g[1] + rng.integers(0, s.n[1]), g[0] + rng.integers(0, s.n[0]))
        du = np.zeros_like(u)
        du[k, j, i] = rng.standard_normal(s.nvar)
        db = dp = None
        if s.magnetic:
            db = np.zeros_like(b)
            db[k, j, i] = rng.standard_normal(3)
            dp = np.zeros_like(psi)
            dp[k, j, i] = rng.standard_normal()
        _, (tu, tb, tp) = tangent.jvp(s, u, b, psi, du, db, dp, dts)
        eps = 1e-6
        outs = []
        for sgn in (1, -1):
            ob = oracle.OracleBlock(s, u + sgn * eps * du, None if b is None else b + sgn * eps * db,
                                    None if psi is None else psi + sgn * eps * dp)
            # seeds sit in the interior only; the guard images follow them through the fill
            ob.fill_guards()
            assert ob.run_fixed(dts) == 0
            ob.fill_guards()
            outs.append(ob)
        fd = (outs[0].u - outs[1].u) / (2 * eps)
        inner = (slice(g[2], g[2] + s.n[2]), slice(g[1], g[1] + s.n[1]), slice(g[0], g[0] + s.n[0]))
        # the tangent seed did not move the guard images: compare after the final
        # guard fill, on the interior
        err = np.max(np.abs(tu[inner] - fd[inner])) / max(np.max(np.abs(fd[inner])), 1e-300)
        worst = max(worst, err)
    assert worst < 1e-6, worst
