"""CPU checks of the oracle itself (no GPU).

The reference ships no golden vectors for the split sweep, so the oracle is
pinned by physics properties that hold bit-for-bit or to round-off:
conservation on periodic boxes, exact symmetry under exchanging axes, GLM
damping and CFL formulas restated independently in numpy.
"""
import ctypes as C
import math

import numpy as np
import pytest

import oracle
from helpers import assert_bitexact, interior, random_state, setup_for
from piernik_b200 import problems

LIMS = ["vanleer", "minmod", "moncen", "superbee", "weno3"]   # weno3: interpol_str = weno3


def totals(setup, ob):
    t = interior(setup, ob.u).reshape(-1, setup.nvar).sum(0)
    if setup.magnetic:
        t = np.concatenate([t, interior(setup, ob.b).reshape(-1, 3).sum(0)])
    return t


@pytest.mark.parametrize("phys", ["hd", "mhd"])
@pytest.mark.parametrize("lim", LIMS)
def test_conservation_periodic(oracle_lib, phys, lim):
    s = setup_for(phys, n=(16, 12, 10), lim=lim)
    u, b, psi = random_state(s, seed=1)
    ob = oracle.OracleBlock(s, u, b, psi)
    t0 = totals(s, ob)
    dt, _ = ob.timestep_raw()
    for d in (0, 1, 2, 2, 1, 0):
        ob.sweep(d, dt, 1.0)
    t1 = totals(s, ob)
    scale = np.abs(interior(s, ob.u)).reshape(-1, s.nvar).sum(0)
    if s.magnetic:
        scale = np.concatenate([scale, np.abs(interior(s, ob.b)).reshape(-1, 3).sum(0)])
    assert np.all(np.abs(t1 - t0) <= 1e-13 * scale)


def _swap_axes(setup, u, b, psi, a1, a2):
    ax = lambda d: 2 - d
    u2 = np.swapaxes(u, ax(a1), ax(a2)).copy()
    beg = 0
    for kind, _ in setup.fluids:
        u2[..., [beg + 1 + a1, beg + 1 + a2]] = u2[..., [beg + 1 + a2, beg + 1 + a1]]
        beg += 4 if kind == "dst" else 5
    if b is None:
        return u2, None, None
    b2 = np.swapaxes(b, ax(a1), ax(a2)).copy()
    b2[..., [a1, a2]] = b2[..., [a2, a1]]
    return u2, b2, np.swapaxes(psi, ax(a1), ax(a2)).copy()


@pytest.mark.parametrize("phys", ["hd", "mhd"])
@pytest.mark.parametrize("lim", LIMS)
@pytest.mark.parametrize("axes", [(0, 1), (0, 2)])
def test_axis_exchange_symmetry_bitexact(oracle_lib, phys, lim, axes):
    """The x sweep of a state equals the y (z) sweep of its x<->y (x<->z)
    transpose bit for bit: the reference's swept component order makes the two
    computations identical operation by operation."""
    a1, a2 = axes
    s = setup_for(phys, n=(12, 12, 12), lim=lim)
    u, b, psi = random_state(s, seed=5)
    A = oracle.OracleBlock(s, u, b, psi)
    B = oracle.OracleBlock(s, *_swap_axes(s, u, b, psi, a1, a2))
    A.sweep(a1, 0.01, 1.3)
    B.sweep(a2, 0.01, 1.3)
    ub, bb, pb = _swap_axes(s, B.u, B.b, B.psi, a1, a2)
    assert_bitexact(A.u, ub, "u")
    if s.magnetic:
        assert_bitexact(A.b, bb, "b")
        assert_bitexact(A.psi, pb, "psi")


def test_uniform_state_is_steady(oracle_lib):
    """A uniform moving MHD state is an exact steady solution of every sweep."""
    s = setup_for("mhd", n=(10, 9, 8), lim="moncen")
    u, b, psi = problems._empty(s)
    problems._set_fluid(s, u, 0, 1.25, 0.3, -0.2, 0.1, 0.6, 0.5 * (0.25 + 0.01 + 0.04))
    b[...] = (0.5, 0.1, -0.2)
    ob = oracle.OracleBlock(s, u, b, psi)
    for d in range(3):
        ob.sweep(d, 0.01, 1.0)
    assert np.allclose(ob.u, u, rtol=1e-14, atol=1e-15)
    assert np.allclose(ob.b, b, rtol=1e-14, atol=1e-15)


def test_timestep_matches_numpy(oracle_lib):
    """timestep_fluid restated in numpy (ion_cs with B, timestep.F90:431-495)."""
    s = setup_for("mhd", n=(11, 7, 5), lim="vanleer")
    u, b, psi = random_state(s, seed=2)
    ob = oracle.OracleBlock(s, u, b, psi)
    dt, c_all = ob.timestep_raw()
    ui, bi = interior(s, u), interior(s, b)
    dn, m, en = ui[..., 0], ui[..., 1:4], ui[..., 4]
    pmag = 0.5 * ((bi[..., 0] ** 2 + bi[..., 1] ** 2) + bi[..., 2] ** 2)
    ek = 0.5 * ((m[..., 0] ** 2 + m[..., 1] ** 2) + m[..., 2] ** 2) / dn
    gam = 5.0 / 3.0
    ps = (en - ek) * (gam - 1.0) + (2.0 - gam) * pmag
    cs = np.sqrt(np.abs((2.0 * pmag + gam * (ps - pmag)) / dn))
    small = np.float64(np.finfo(np.float32).tiny)
    c = np.maximum(np.abs(m / dn[..., None]) + cs[..., None], small)
    dt_np = s.cfl * min(s.dl[d] / c[..., d].max() for d in range(3))
    assert dt == dt_np
    assert c_all == c.max()


def test_glm_formulas(oracle_lib):
    """update_chspeed / glmdamping with ch_grid (hdc.F90:112-119, 310-330)."""
    s = setup_for("mhd", n=(8, 8, 4), lim="vanleer")
    u, b, psi = random_state(s, seed=3)
    ob = oracle.OracleBlock(s, u, b, psi)
    dt = 0.0123
    ch = ob.chspeed(dt)
    mdl = min(s.dl)
    assert ch == (s.cfl_glm * mdl) / dt
    assert ob.glm_fac(dt, ch) == math.exp(-((s.glm_alpha * ch) / (mdl / dt)))


def test_run_clamps_and_counts(oracle_lib):
    """time_step clamps: first step unclamped for dt_initial=-1, then
    dt <= 2*dt_old, and the last step is cut to reach tend (timestep.F90:200-224)."""
    setup, u, b, psi = problems.sedov(n=16)
    setup = setup.replace(tend=0.02)
    ob = oracle.OracleBlock(setup, u, b, psi)
    ob.run(1)
    dt0 = ob.state.dt
    assert ob.state.nstep == 1 and ob.state.t == 2 * dt0
    prev = dt0
    for _ in range(200):
        if not ob.state.t < setup.tend:
            break
        ob.run(1)
        assert ob.state.dt <= 2.0 * prev
        prev = ob.state.dt
    assert ob.state.t >= setup.tend * (1 - 1e-12)


def test_sedov_blast_expands(oracle_lib):
    """Sedov: the shock moves outward and stays centred (symmetric deposit)."""
    setup, u, b, psi = problems.sedov(n=24)
    ob = oracle.OracleBlock(setup, u, b, psi)
    ob.run(20)
    rho = interior(setup, ob.u)[..., 0]
    assert rho.max() > 1.5
    c = setup.n[0] // 2
    prof = rho[c, c, :]
    assert np.allclose(prof, prof[::-1], rtol=1e-12)
    assert abs(rho.sum() * np.prod(setup.dl) - 8.0) < 1e-10


@pytest.mark.parametrize("fluids,mag", [
    ([("ion", 5 / 3), ("neu", 1.4)], True),       # HLLD for both fluids, neutral with B = 0
    ([("neu", 1.4), ("dst", -1.0)], False),       # HLLC with pressureless dust
])
def test_multifluid_solve_conserves(oracle_lib, fluids, mag):
    """Several fluids in one pencil solve (riemann_wrap loops over fluids,
    hlld.F90:62-155); mass and momentum of every fluid are conserved."""
    from piernik_b200.config import Setup
    s = Setup(n=(10, 8, 6), fluids=fluids, magnetic=mag, limiter="moncen", limiter_b="moncen",
              xmin=(0, 0, 0), xmax=(1, 0.8, 0.6))
    u, b, psi = problems.random_state(s, seed=4)
    ob = oracle.OracleBlock(s, u, b, psi)
    m0 = interior(s, ob.u).reshape(-1, s.nvar).sum(0)
    for d in range(3):
        ob.sweep(d, 0.005, 1.0)
    m1 = interior(s, ob.u).reshape(-1, s.nvar).sum(0)
    scale = np.abs(interior(s, ob.u)).reshape(-1, s.nvar).sum(0)
    assert np.all(np.abs(m1 - m0) <= 1e-13 * scale)


def test_dust_in_hlld_diverging_flow_is_nan(oracle_lib):
    """Faithful-restatement check: with B present every fluid goes through
    riemann_hlld, and for dust (gamma < 0, c_fast = 0) in a diverging flow
    sl = vx_l gives dn_l = 0, so b_ccl(x)/dn_l at hlld.F90:381 is 0/0 and the
    momentum flux is NaN.  The reference computes exactly this."""
    from piernik_b200.config import Setup
    s = Setup(n=(8, 4, 4), fluids=[("ion", 5 / 3), ("dst", -1.0)], magnetic=True, limiter="minmod",
              limiter_b="minmod", xmin=(0, 0, 0), xmax=(1, 0.5, 0.5))
    u, b, psi = problems.random_state(s, seed=1)
    g = s.guards
    x = np.arange(s.ext[0]) - g[0]
    u[..., 5] = 1.0
    u[..., 6] = np.where(x < s.n[0] // 2, -0.1, 0.1)[None, None, :]    # dust diverges at the centre
    ob = oracle.OracleBlock(s, u, b, psi)
    ob.solve_cg(0, 1, 0.001, 1.0)
    assert np.isnan(interior(s, ob.u)[..., 5:9]).any()
    assert not np.isnan(interior(s, ob.u)[..., 0:5]).any()


def test_cfl_redo_without_violation_equals_none(oracle_lib):
    """cflcontrol = redo changes nothing when no step violates cfl_max."""
    from piernik_b200 import problems
    s, u, b, psi = problems.sedov(n=16)
    runs = []
    for mode in ("none", "redo"):
        ob = oracle.OracleBlock(s.replace(cfl=0.7, cflcontrol=mode), u, b, psi)
        assert ob.run(12) == 0
        runs.append(ob)
    assert runs[1].state.redone == 0
    assert np.array_equal(runs[0].u.view(np.uint64), runs[1].u.view(np.uint64))
    assert runs[0].state.t == runs[1].state.t


def test_cfl_redo_repeats_violating_steps(oracle_lib):
    """At cfl = 0.9 the early Sedov blast speeds up faster than cfl_max allows
    (stepcfl = c_new/c_old * cfl > 0.95): those steps are redone with half
    the time step (timestep_retry.F90, timestep.F90:317-360)."""
    from piernik_b200 import problems
    s, u, b, psi = problems.sedov(n=24)
    s = s.replace(cfl=0.9, cflcontrol="redo")
    ob = oracle.OracleBlock(s, u, b, psi)
    assert ob.run(30) == 0
    st = ob.state
    assert st.redone > 0
    assert st.nstep == 30 - st.redone
    assert st.stepcfl <= oracle.lib().o_cfl_max(C.byref(ob.cfg))
    assert st.dt_cur_shrink == 1.0


def test_cfl_flex_repeats_with_flexible_shrink(oracle_lib):
    """cflcontrol = flex: the same retries as redo, with dt_cur_shrink =
    cfl_max / stepcfl on the first retry (x dt_shrink from the second on,
    timestep.F90:81-84,347-351) instead of dt_shrink**attempt; a retried step
    then lands at stepcfl = cfl_max, so it is not retried again."""
    from piernik_b200 import problems
    s, u, b, psi = problems.sedov(n=24)
    runs = {}
    for mode in ("redo", "flex"):
        ob = oracle.OracleBlock(s.replace(cfl=0.9, cflcontrol=mode), u, b, psi)
        assert ob.run(30) == 0
        runs[mode] = ob
    fl, rd = runs["flex"].state, runs["redo"].state
    assert fl.redone > 0 and rd.redone > 0
    assert fl.nstep == 30 - fl.redone
    assert not np.array_equal(runs["flex"].u.view(np.uint64), runs["redo"].u.view(np.uint64))
    assert fl.stepcfl <= oracle.lib().o_cfl_max(C.byref(runs["flex"].cfg))


def test_cfl_auto_follows_its_recurrence(oracle_lib):
    """cflcontrol = auto: every main time step is the CFL step (with the
    dt_old x dt_max_grow clamp) times cfl_c, where cfl_c = min(1, (cfl_c +
    min(1, stepcfl_old / stepcfl * dt / dt_old)) / 2) and stepcfl =
    c_all / c_all_old * cfl (timestep.F90:368-405); restated here step by step
    from the oracle's own CFL reduction on the state before each step."""
    from piernik_b200 import problems
    s, u, b, psi = problems.sedov(n=16)
    s = s.replace(cfl=0.7, cflcontrol="auto")
    ob = oracle.OracleBlock(s, u, b, psi)
    cfl_c, stepcfl, c_old, dt_prev = 1.0, 0.0, 0.0, 0.0
    shrunk = 0
    for k in range(14):
        dt_raw, c_all = ob.timestep_raw()
        dt = dt_raw
        if k >= 1 and dt_prev > 0.0:
            dt = min(dt, dt_prev * s.dt_max_grow)
        st_old = stepcfl
        stepcfl = s.cfl
        if c_old > 0.0:
            stepcfl = (c_all / c_old) * s.cfl
        else:
            st_old = s.cfl
        if stepcfl > 0.0 and dt_prev > 0.0:
            r = min(1.0, ((st_old / stepcfl) * dt) / dt_prev)
            cfl_c = min(1.0, 0.5 * (cfl_c + r))
            dt = dt * cfl_c
        else:
            cfl_c = 1.0
        assert ob.run(1) == 0
        assert ob.state.dt == dt and ob.state.cfl_c == cfl_c and ob.state.stepcfl == stepcfl, k
        shrunk += cfl_c < 1.0
        c_old, dt_prev = c_all, dt
    assert shrunk > 0


@pytest.mark.parametrize("phys", ["mhd", "hd-neu"])
def test_gas_chspeed_restated(oracle_lib, phys):
    """ch_grid = .false.: chspeed is the maximum over the block's cells of
    point_chspeed (hdc.F90:197-268), restated here with numpy in the same
    operation order, bit for bit."""
    from helpers import random_state, setup_for
    s = setup_for("mhd" if phys == "mhd" else "hd", n=(12, 10, 8), lim="moncen").replace(ch_grid=False)
    u, b, psi = random_state(s, seed=3)
    ob = oracle.OracleBlock(s, u, b, psi)
    got = oracle.lib().o_chspeed(C.byref(ob.cfg), C.byref(ob.blk), 0.01)
    g, n = s.guards, s.n
    cut = lambda a: a[g[2]:g[2] + n[2], g[1]:g[1] + n[1], g[0]:g[0] + n[0]]
    U = cut(u)
    dn, m, E = U[..., 0], [U[..., 1], U[..., 2], U[..., 3]], U[..., 4]
    gam = s.fluids[0][1]
    ek = (0.5 * ((m[0] * m[0] + m[1] * m[1]) + m[2] * m[2])) / dn
    best = np.float64(1.1754943508222875e-38)
    if s.magnetic:
        B = cut(b)
        pmag = 0.5 * ((B[..., 0] * B[..., 0] + B[..., 1] * B[..., 1]) + B[..., 2] * B[..., 2])
        pgam = ((0.5 * gam) * (gam - 1.0)) * ((E - ek) - pmag)
        for d in range(3):
            sp = pgam + pmag
            c = s.cfl_glm * (np.abs(m[d] / dn) + np.sqrt((sp + np.sqrt(sp * sp - (2.0 * pgam) * (B[..., d] * B[..., d]))) / dn))
            best = max(best, c.max())
    else:
        pgam = ((0.5 * gam) * (gam - 1.0)) * (E - ek)
        for d in range(3):
            best = max(best, (s.cfl_glm * (np.abs(m[d] / dn) + np.sqrt((2.0 * pgam) / dn))).max())
    assert got == best


def test_sedov_shock_follows_similarity_solution(oracle_lib):
    """Sedov-Taylor: the blast front (peak of the spherically averaged
    density) sits at R = xi0 (E t^2 / rho)^(1/5), xi0 = 1.1517 for gamma =
    5/3 in 3D, within 10 % at 48^3, and R grows as t^(2/5) between t = 0.05
    and 0.1 within 5 % (the physics check of the restated split solver)."""
    radii = []
    for tend in (0.05, 0.1):
        setup, u, b, psi = problems.sedov(n=48)
        setup = setup.replace(tend=tend)
        ob = oracle.OracleBlock(setup, u, b, psi)
        ob.run(5000)
        assert abs(ob.state.t - tend) <= 1e-12
        rho = interior(setup, ob.u)[..., 0]
        n, dx = setup.n[0], setup.dl[0]
        c = (np.arange(n) + 0.5) * dx - 1.0
        Z, Y, X = np.meshgrid(c, c, c, indexing="ij")
        R = np.sqrt(X ** 2 + Y ** 2 + Z ** 2).ravel()
        edges = np.arange(0.0, 1.0, dx / 2)
        k = np.digitize(R, edges)
        cnt = np.bincount(k, minlength=len(edges) + 1)[1:len(edges)]
        tot = np.bincount(k, weights=rho.ravel(), minlength=len(edges) + 1)[1:len(edges)]
        prof = np.where(cnt > 0, tot / np.maximum(cnt, 1), 0.0)
        r_shock = 0.5 * (edges[1:] + edges[:-1])[np.argmax(prof)]
        r_theory = 1.15167 * (1.0 * tend ** 2 / 1.0) ** 0.2
        assert 0.9 < r_shock / r_theory < 1.1, (tend, r_shock, r_theory)
        radii.append(r_shock)
    assert abs(radii[1] / radii[0] / 2.0 ** 0.4 - 1.0) < 0.05, radii
