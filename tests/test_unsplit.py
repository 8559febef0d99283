"""The unsplit scheme (solver_str = 'unsplit', src/scheme/unsplit_schemes).

CPU: the oracle's restatement conserves every conserved quantity on a
periodic box and keeps a uniform moving state steady; time steps advance by
one dt per step with the unsplit end-of-run clamp.  GPU: the library's
unsplit stages and runs equal the oracle bit for bit (guard cells included)
for HD and MHD, 2D and 3D, limited-linear and WENO3 reconstruction."""
import numpy as np
import pytest

import oracle
from helpers import assert_bitexact, interior, random_state, setup_for, smooth_state
from piernik_b200 import problems


def useup(phys, n=(16, 12, 10), lim="vanleer", **kw):
    kw.setdefault("cfl", 0.3)
    kw.setdefault("cfl_glm", 0.3)
    return setup_for(phys, n=n, lim=lim, solver="unsplit", **kw)


@pytest.mark.parametrize("phys", ["hd", "mhd"])
@pytest.mark.parametrize("n", [(16, 12, 10), (16, 12, 1)])
def test_unsplit_oracle_conserves(oracle_lib, phys, n):
    s = useup(phys, n=n)
    ob = oracle.OracleBlock(s, *smooth_state(s, seed=1))
    ob.fill_guards()
    tot = lambda: interior(s, ob.u).reshape(-1, s.nvar).sum(0)
    scale = np.abs(interior(s, ob.u)).reshape(-1, s.nvar).sum(0)
    t0 = tot()
    assert ob.run(4) == 0
    assert ob.state.nstep == 4 and ob.state.t > 0
    assert np.all(np.abs(tot() - t0) <= 1e-12 * scale)


def test_unsplit_uniform_state_is_steady(oracle_lib):
    s = useup("mhd", n=(10, 9, 8), lim="moncen")
    u, b, psi = problems._empty(s)
    problems._set_fluid(s, u, 0, 1.25, 0.3, -0.2, 0.1, 0.6, 0.5 * (0.25 + 0.01 + 0.04))
    b[...] = (0.5, 0.1, -0.2)
    ob = oracle.OracleBlock(s, u, b, psi)
    ob.run(2)
    assert np.allclose(ob.u, u, rtol=1e-14, atol=1e-15)
    assert np.allclose(ob.b, b, rtol=1e-14, atol=1e-15)


def test_unsplit_one_dt_per_step_and_end_clamp(oracle_lib):
    """One dt per step (t += dt), and the last step reaches tend with
    dt <= tend - t (timestep.F90:221-225) instead of half of it."""
    s = useup("hd", n=(12, 12, 12)).replace(tend=0.05)
    ob = oracle.OracleBlock(s, *smooth_state(s, seed=2))
    ob.fill_guards()
    ob.run(1)
    assert ob.state.t == ob.state.dt
    for _ in range(100):
        if not ob.state.t < s.tend:
            break
        ob.run(1)
    assert abs(ob.state.t - s.tend) <= 1e-12


# ---- GPU parity --------------------------------------------------------------
CASES = [("hd", (16, 12, 10), "vanleer"), ("mhd", (16, 12, 10), "moncen"), ("mhd", (16, 12, 1), "vanleer"),
         ("mhd", (16, 12, 10), "weno3"), ("hd", (12, 10, 8), "minmod"),
         ("mhd", (8, 100, 6), "vanleer")]          # y pencils in chunks (fewer than 4 whole ones fit a CTA)


@pytest.mark.gpu
@pytest.mark.parametrize("phys,n,lim", CASES)
def test_unsplit_matches_oracle(gpu_lib, phys, n, lim):
    from piernik_b200.sim import Simulation
    s = useup(phys, n=n, lim=lim)
    u, b, psi = random_state(s, seed=7)
    ob = oracle.OracleBlock(s, u, b, psi)
    ob.fill_guards()
    sim = Simulation(s)
    sim.upload(ob.u, ob.b, ob.psi)
    sim.run(3)
    ob.run(3)
    gu, gb, gp = sim.download()
    assert_bitexact(gu, ob.u, "u")
    if s.magnetic:
        assert_bitexact(gb, ob.b, "b")
        assert_bitexact(gp, ob.psi, "psi")
    st = sim.time_state
    assert (st.t, st.dt, st.nstep, st.chspeed) == (ob.state.t, ob.state.dt, ob.state.nstep, ob.state.chspeed)
    sim.close()


@pytest.mark.gpu
def test_unsplit_euler_and_outflow(gpu_lib):
    """First-order (EULER) stages and outflow boundaries, HD."""
    from piernik_b200.config import BND_OUT
    from piernik_b200.sim import Simulation
    s = useup("hd", n=(16, 12, 10), integration_order=1).replace(bnd=((BND_OUT, BND_OUT),) * 3)
    ob = oracle.OracleBlock(s, *smooth_state(s, seed=3))
    ob.fill_guards()
    sim = Simulation(s)
    sim.upload(ob.u)
    sim.run(3)
    ob.run(3)
    assert_bitexact(sim.download()[0], ob.u, "u")
    sim.close()


@pytest.mark.gpu
@pytest.mark.parametrize("phys,lim,order,periodic", [("mhd", "moncen", 2, True), ("hd", "vanleer", 2, False),
                                                     ("hd", "minmod", 1, True), ("mhd", "weno3", 2, True)])
def test_unsplit_tiled_domain_equals_one_block(gpu_lib, phys, lim, order, periodic):
    """Blocks of one level tiling the domain (the uh stage array exchanged
    after the first stage, u after the second, unsplit_sweeps.F90:182)
    evolve exactly like the oracle's single block."""
    from test_gpu_blocks import exact_dl, interior_of, run_tiled, tiles
    from piernik_b200.config import BND_OUT, BND_PER
    bnd = ((BND_PER, BND_PER),) * 3 if periodic else ((BND_OUT, BND_OUT), (BND_PER, BND_PER), (BND_PER, BND_PER))
    n = (40, 36, 28) if phys == "mhd" else (40, 20, 16)
    full = exact_dl(useup(phys, n=n, lim=lim, integration_order=order).replace(bnd=bnd))
    state = random_state(full, seed=3)
    ob = oracle.OracleBlock(full, *state)
    ob.fill_guards()
    ob.run(3)
    blocks = tiles([16, 24], [20, 16], [12, 16]) if phys == "mhd" else tiles([12, 16, 12], [20], [8, 8])
    st0 = tuple(x.copy() if x is not None else None for x in (ob.u, ob.b, ob.psi))
    fresh = oracle.OracleBlock(full, *state)
    fresh.fill_guards()
    got, st = run_tiled(full, (fresh.u, fresh.b, fresh.psi), blocks, (periodic, True, True), 3, bnd_x=BND_OUT)
    assert (st.t, st.dt, st.nstep) == (ob.state.t, ob.state.dt, ob.state.nstep)
    for (nn, off), arrs in zip(blocks, got):
        s = full.replace(n=nn)
        for k, name in enumerate(("u", "b", "psi")):
            if arrs[k] is None:
                continue
            assert_bitexact(interior_of(s, arrs[k], nn, (0, 0, 0)), interior_of(full, st0[k], nn, off),
                            f"{phys} block {off} {name}")
