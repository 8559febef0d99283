"""Parity of the CUDA path (through the C ABI) with the CPU oracle.

The bar is bit-for-bit equality: the kernels are built with --fmad=false and
keep the reference's operation order, so every double must match the oracle's.
"""
import numpy as np
import pytest

import oracle
from helpers import assert_bitexact, interior, random_state, setup_for
from piernik_b200 import problems
from piernik_b200._lib import PK_EULER, PK_RK2_1, PK_RK2_2, PK_ST_DN_NEGATIVE, PK_ST_TIMEOUT, PK_VARIANT_STAGED
from piernik_b200.config import BND_OUT, BND_PER, BND_REF
from piernik_b200.sim import Simulation

pytestmark = pytest.mark.gpu

LIMS = ["vanleer", "minmod", "moncen", "superbee", "weno3"]   # weno3: interpol_str = weno3


def both(setup, seed=0):
    u, b, psi = random_state(setup, seed)
    ob = oracle.OracleBlock(setup, u, b, psi)
    sim = Simulation(setup)
    sim.upload(u, b, psi)
    return ob, sim


def compare(ob, sim, what, full=True):
    u, b, psi = sim.download()
    s = ob.setup
    if full:
        assert_bitexact(u, ob.u, what + " u")
        if s.magnetic:
            assert_bitexact(b, ob.b, what + " b")
            assert_bitexact(psi, ob.psi, what + " psi")
    else:
        assert_bitexact(interior(s, u), interior(s, ob.u), what + " u")
        if s.magnetic:
            assert_bitexact(interior(s, b), interior(s, ob.b), what + " b")
            assert_bitexact(interior(s, psi), interior(s, ob.psi), what + " psi")


@pytest.mark.parametrize("phys", ["hd", "mhd"])
@pytest.mark.parametrize("lim", LIMS)
def test_solve_cg_stage_bitexact(gpu_lib, oracle_lib, phys, lim):
    """pk_solve_cg == solve_cg_riemann for every direction and RK stage, guard cells included."""
    s = setup_for(phys, n=(12, 10, 8), lim=lim, limb="moncen" if lim != "moncen" else "minmod")
    ob, sim = both(s, seed=11)
    dt, ch = 0.013, 1.7
    for ddim in (1, 2, 3):
        for istep, oi in ((PK_RK2_1, 1), (PK_RK2_2, 2)):
            sim.solve_cg(ddim, istep, dt, ch)
            ob.solve_cg(ddim - 1, oi, dt, ch)
            compare(ob, sim, f"solve_cg d{ddim} s{istep}")


@pytest.mark.parametrize("phys", ["hd", "mhd"])
def test_solve_cg_euler(gpu_lib, oracle_lib, phys):
    s = setup_for(phys, n=(10, 9, 7), lim="moncen", integration_order=1)
    ob, sim = both(s, seed=3)
    for ddim in (1, 2, 3):
        sim.solve_cg(ddim, PK_EULER, 0.01, 1.2)
        ob.solve_cg(ddim - 1, 1, 0.01, 1.2)
        compare(ob, sim, f"euler d{ddim}")


@pytest.mark.parametrize("phys", ["hd", "mhd"])
@pytest.mark.parametrize("lim", LIMS)
def test_fused_sweep_bitexact(gpu_lib, oracle_lib, phys, lim):
    """The fused two-stage sweep of a periodic block equals stage/exchange/stage."""
    s = setup_for(phys, n=(20, 14, 11), lim=lim)
    ob, sim = both(s, seed=5)
    dt, ch = 0.011, 1.3
    for d in (0, 1, 2, 2, 1, 0):
        sim.sweep(d + 1, dt, ch)
        ob.sweep(d, dt, ch)
    compare(ob, sim, "fused sweeps")


@pytest.mark.parametrize("tile", [(1, 8, 3), (3, 16, 4), (4, 40, 1), (2, 64, 0), (8, 24, 2), (2, 56, 5), (7, 24, 6),
                                  (1, 50, 6)])
def test_fused_tiles_agree(gpu_lib, oracle_lib, tile):
    """Tile shapes (pencils per CTA, cells per chunk, launch-bound variant) do
    not change any bit."""
    s = setup_for("mhd", n=(50, 37, 29), lim="moncen")
    ob, sim = both(s, seed=9)
    for d in range(3):
        sim.set_tile(d, *tile)
    dt, ch = 0.009, 1.1
    for d in (0, 1, 2):
        sim.sweep(d + 1, dt, ch)
        ob.sweep(d, dt, ch)
    compare(ob, sim, f"tile {tile}")


@pytest.mark.parametrize("phys,n,lim", [("mhd", (50, 37, 29), "moncen"), ("hd", (48, 31, 20), "vanleer"),
                                         ("mhd", (64, 48, 1), "moncen"), ("mhd", (36, 30, 22), "superbee"),
                                         ("hd", (8, 8, 8), "minmod")])
def test_staged_sweeps_bitexact(gpu_lib, oracle_lib, phys, n, lim):
    """The TMA-staged whole-pencil kernel (PK_VARIANT_STAGED: two pencils per
    CTA, the box loaded and stored by bulk-tensor copies) along every
    direction, with an odd number of pencils across (the last CTA sweeps one)
    and pencils shorter than a warp multiple, equals the oracle bit for bit."""
    s = setup_for(phys, n=n, lim=lim)
    ob, sim = both(s, seed=13)
    for d in range(3):
        sim.set_tile(d, 2, 0, PK_VARIANT_STAGED)
    dt, ch = 0.009, 1.2
    for d in (0, 1, 2, 2, 1, 0):
        if n[d] > 1:
            sim.sweep(d + 1, dt, ch)
            ob.sweep(d, dt, ch)
    compare(ob, sim, "staged sweeps")
    assert not (sim.status() & PK_ST_TIMEOUT)


def test_staged_run_with_graph(gpu_lib, oracle_lib):
    """Whole main-loop steps with the staged kernel on y and z, replayed from a CUDA graph."""
    setup, u, b, psi = problems.mhd_turbulence(n=32, seed=6)
    ob = oracle.OracleBlock(setup, u, b, psi)
    sim = Simulation(setup)
    sim.upload(u, b, psi)
    sim.set_tile(1, 2, 0, PK_VARIANT_STAGED)
    sim.set_tile(2, 2, 0, PK_VARIANT_STAGED)
    sim.use_graph(True)
    sim.run(3)
    ob.run(3)
    compare(ob, sim, "staged run")


def test_stage_path_long_pencil(gpu_lib, oracle_lib):
    """Pencils longer than one CTA tile go through the chunked out-of-place stage."""
    s = setup_for("mhd", n=(400, 6, 5), lim="vanleer", integration_order=1)
    ob, sim = both(s, seed=2)
    for ddim in (1, 2, 3):
        sim.solve_cg(ddim, PK_EULER, 0.004, 1.0)
        ob.solve_cg(ddim - 1, 1, 0.004, 1.0)
    compare(ob, sim, "long pencil")


@pytest.mark.parametrize("bnd", [BND_OUT, BND_REF])
def test_nonperiodic_hd_sweeps(gpu_lib, oracle_lib, bnd):
    """Outflow / reflecting boundaries take the stage + guard-refresh path."""
    s = setup_for("hd", n=(16, 12, 10), lim="moncen", bnd=((bnd, bnd), (BND_PER, BND_PER), (bnd, BND_OUT)))
    ob, sim = both(s, seed=4)
    for d in (0, 1, 2, 2, 1, 0):
        sim.sweep(d + 1, 0.01, 0.0)
        ob.sweep(d, 0.01, 0.0)
    compare(ob, sim, "non-periodic")


@pytest.mark.parametrize("phys", ["hd", "mhd"])
def test_timestep_raw_bitexact(gpu_lib, oracle_lib, phys):
    s = setup_for(phys, n=(24, 17, 9), lim="vanleer")
    ob, sim = both(s, seed=8)
    dt_g, c_g = sim.timestep_raw()
    dt_o, c_o = ob.timestep_raw()
    assert dt_g == dt_o and c_g == c_o


def run_pair(setup, u, b, psi, nsteps):
    ob = oracle.OracleBlock(setup, u, b, psi)
    sim = Simulation(setup)
    sim.upload(u, b, psi)
    ob.run(nsteps)
    sim.run(nsteps)
    return ob, sim


def test_run_sedov_hd_bitexact(gpu_lib, oracle_lib):
    """Sedov blast (HLLC, van Leer, CFL 0.7), 10 pairs of steps through pk_run."""
    setup, u, b, psi = problems.sedov(n=24)
    ob, sim = run_pair(setup, u, b, psi, 10)
    st = sim.time_state
    assert st.nstep == ob.state.nstep == 10
    assert st.t == ob.state.t and st.dt == ob.state.dt
    compare(ob, sim, "sedov run")


def test_run_mhd_turbulence_bitexact(gpu_lib, oracle_lib):
    """Decaying MHD turbulence (HLLD + GLM, moncen, CFL 0.5), 10 pairs of steps."""
    setup, u, b, psi = problems.mhd_turbulence(n=20, seed=3)
    ob, sim = run_pair(setup, u, b, psi, 10)
    st = sim.time_state
    assert st.t == ob.state.t and st.dt == ob.state.dt and st.chspeed == ob.state.chspeed
    compare(ob, sim, "mhd run")


def test_run_orszag_tang_2d_bitexact(gpu_lib, oracle_lib):
    """2D run (no z extent, so no z sweep and no z guard cells)."""
    setup, u, b, psi = problems.orszag_tang(n=32, seed=1)
    ob, sim = run_pair(setup, u, b, psi, 8)
    compare(ob, sim, "orszag-tang")


def test_status_flags_negative_density(gpu_lib, oracle_lib):
    """A negative density is reported through pk_status, never by a trap."""
    s = setup_for("hd", n=(8, 8, 8), lim="minmod")
    u, b, psi = random_state(s, seed=1)
    g = s.guards
    u[g[2] + 3, g[1] + 3, g[0] + 3, 0] = -0.2
    sim = Simulation(s)
    sim.upload(u, b, psi)
    sim.sweep(1, 0.001, 0.0)
    assert sim.status() & PK_ST_DN_NEGATIVE
    assert sim.status() == 0


def test_soa_layout_roundtrip(gpu_lib):
    s = setup_for("mhd", n=(9, 8, 7))
    u, b, psi = random_state(s, seed=6)
    sim = Simulation(s)
    sim.upload(u, b, psi)
    su, sb, sp = sim.download(layout=1)
    assert_bitexact(np.moveaxis(su, 0, -1), u, "soa u")
    assert_bitexact(np.moveaxis(sb, 0, -1), b, "soa b")
    assert_bitexact(sp, psi, "soa psi")


def test_autotune_keeps_state(gpu_lib, oracle_lib):
    """The autotuner restores the state it times on and keeps results bit-exact."""
    from piernik_b200.autotune import autotune
    setup, u, b, psi = problems.mhd_turbulence(n=24, seed=5)
    sim = Simulation(setup)
    sim.upload(u, b, psi)
    best = autotune(sim, reps=1)
    assert set(best) == {0, 1, 2}
    ob = oracle.OracleBlock(setup, u, b, psi)
    ob.run(3)
    sim.run(3)
    compare(ob, sim, "after autotune")


def _multi(blocks_data, nsteps, batched=True, graph=False, batch_L=0, batch_V=-1):
    setup0 = blocks_data[0][0]
    sim = Simulation(setup0)
    for s, u, b, psi in blocks_data[1:]:
        sim.add_block(s)
    for i, (s, u, b, psi) in enumerate(blocks_data):
        sim.upload(u, b, psi, block=i)
    if batched:
        sim.set_batch(True, batch_L, batch_V)
    if graph:
        sim.use_graph(True)
    obs = [oracle.OracleBlock(s, u, b, psi) for s, u, b, psi in blocks_data]
    st = oracle.run_multi(obs, nsteps)
    sim.run(nsteps)
    ts = sim.time_state
    assert ts.t == st.t and ts.dt == st.dt and ts.nstep == st.nstep
    for i, ob in enumerate(obs):
        gu, gb, gp = sim.download(block=i)
        assert_bitexact(gu, ob.u, f"block {i} u")
        if ob.setup.magnetic:
            assert_bitexact(gb, ob.b, f"block {i} b")
            assert_bitexact(gp, ob.psi, f"block {i} psi")


@pytest.mark.parametrize("fluids,mag", [
    ((("ion", 5 / 3),), True),
    ((("ion", 5 / 3), ("neu", 1.4)), True),
    ((("ion", 5 / 3), ("neu", 1.4), ("dst", -1.0)), True),
    ((("neu", 1.4), ("dst", -1.0)), False),
    ((("neu", 1.4),), False),
])
def test_batched_uneven_blocks_bitexact(gpu_lib, oracle_lib, fluids, mag):
    """Independent blocks of uneven sizes (3 refinement levels, one global dt)
    swept in one persistent launch per direction, against the oracle's leaves loop."""
    data = problems.batched_blocks(nblocks=6, seed=3, sizes=(8, 12, 16, 20), fluids=fluids, magnetic=mag, n0=16)
    _multi(data, 4)


def test_batched_graph_bitexact(gpu_lib, oracle_lib):
    """The same with each step's sweeps replayed from one captured CUDA graph."""
    data = problems.batched_blocks(nblocks=5, seed=7, sizes=(8, 16, 24), n0=16)
    _multi(data, 5, graph=True, batch_L=16, batch_V=3)


def test_single_block_graph_and_forced_batch(gpu_lib, oracle_lib):
    setup, u, b, psi = problems.mhd_turbulence(n=24, seed=4)
    _multi([(setup, u, b, psi)], 4, batched=False, graph=True)
    _multi([(setup, u, b, psi)], 3, batched=True, graph=False)


@pytest.mark.parametrize("cfl", [0.7, 0.9])
def test_cfl_redo_matches_oracle(gpu_lib, oracle_lib, cfl):
    """cflcontrol = redo: steps whose effective CFL exceeds cfl_max are redone
    from the saved state with a shrunk dt; the whole history (state, t, dt,
    nstep, retries) equals the oracle's."""
    s, u, b, psi = problems.sedov(n=24)
    s = s.replace(cfl=cfl, cflcontrol="redo")
    ob = oracle.OracleBlock(s, u, b, psi)
    sim = Simulation(s)
    sim.upload(u, b, psi)
    assert ob.run(30) == 0
    sim.run(30)
    st, ost = sim.time_state, ob.state
    for f in ("t", "dt", "dt_old", "c_all", "dt_full", "c_all_old", "dt_cur_shrink", "stepcfl", "t_saved"):
        assert getattr(st, f) == getattr(ost, f), f
    assert (st.nstep, st.redone, st.repeat_step, st.tstep_attempt) == (ost.nstep, ost.redone, ost.repeat, ost.tstep_attempt)
    assert (st.redone > 0) == (cfl == 0.9)
    compare(ob, sim, f"redo cfl={cfl}")
    sim.close()


@pytest.mark.parametrize("recipe", ["mhd", "ot", "batched", "sedov"])
def test_weno3_runs_bitexact(gpu_lib, oracle_lib, recipe):
    """interpol_str = 'weno3' (interpolations.F90:210-337) on whole runs:
    fused single block (MHD turbulence, 2D Orszag-Tang), the batched sweep
    over uneven 3-fluid blocks, and the Sedov blast with outflow boundaries
    (per-stage path with pencil ends)."""
    if recipe == "batched":
        data = problems.batched_blocks(nblocks=5, seed=9, sizes=(8, 12, 16), n0=16)
        data = [(s.replace(interpolation="weno3"), u, b, psi) for s, u, b, psi in data]
        _multi(data, 3)
        return
    if recipe == "mhd":
        setup, u, b, psi = problems.mhd_turbulence(n=20, seed=5)
    elif recipe == "ot":
        setup, u, b, psi = problems.orszag_tang(n=32, seed=2)
    else:
        setup, u, b, psi = problems.sedov(n=20)
        setup = setup.replace(bnd=((BND_OUT, BND_OUT),) * 3)
    setup = setup.replace(interpolation="weno3")
    ob, sim = run_pair(setup, u, b, psi, 6)
    st = sim.time_state
    assert st.t == ob.state.t and st.dt == ob.state.dt
    compare(ob, sim, f"weno3 {recipe}")


@pytest.mark.parametrize("mode", ["flex", "auto"])
def test_cfl_flex_auto_match_oracle(gpu_lib, oracle_lib, mode):
    """cflcontrol = flex (retries with dt_cur_shrink = cfl_max / stepcfl) and
    auto (cfl_auto's dt x cfl_c in every main time step): the whole history
    equals the oracle's."""
    s, u, b, psi = problems.sedov(n=24)
    s = s.replace(cfl=0.9 if mode == "flex" else 0.7, cflcontrol=mode)
    ob = oracle.OracleBlock(s, u, b, psi)
    sim = Simulation(s)
    sim.upload(u, b, psi)
    assert ob.run(30) == 0
    sim.run(30)
    st, ost = sim.time_state, ob.state
    for f in ("t", "dt", "dt_old", "c_all", "dt_full", "c_all_old", "dt_cur_shrink", "stepcfl", "cfl_c"):
        assert getattr(st, f) == getattr(ost, f), f
    assert (st.nstep, st.redone) == (ost.nstep, ost.redone)
    if mode == "flex":
        assert st.redone > 0
    else:
        assert st.cfl_c < 1.0 or st.nstep == 30
    compare(ob, sim, f"cflcontrol = {mode}")
    sim.close()


@pytest.mark.parametrize("case", ["split-mhd", "split-2d", "unsplit-mhd", "batched-3fluid"])
def test_gas_chspeed_matches_oracle(gpu_lib, oracle_lib, case):
    """ch_grid = .false.: chspeed is the maximum of point_chspeed over the
    leaf cells (a device reduction), and with it the GLM fluxes and damping."""
    if case == "batched-3fluid":
        data = problems.batched_blocks(nblocks=5, seed=7, sizes=(8, 16, 24), n0=16)
        data = [(st.replace(ch_grid=False), u, b, psi) for st, u, b, psi in data]
        _multi(data, 3)
        return
    if case == "split-2d":
        s, u, b, psi = problems.orszag_tang(n=32, seed=1)
    else:
        s, u, b, psi = problems.mhd_turbulence(n=20, seed=3)
    s = s.replace(ch_grid=False)
    if case.startswith("unsplit"):
        s = s.replace(solver="unsplit", cfl=0.3, cfl_glm=0.3)
    ob, sim = oracle.OracleBlock(s, u, b, psi), Simulation(s)
    sim.upload(u, b, psi)
    ob.run(4)
    sim.run(4)
    st = sim.time_state
    assert st.chspeed == ob.state.chspeed and st.t == ob.state.t
    assert st.chspeed != (s.cfl_glm * min(s.dl[d] for d in range(3) if s.n[d] > 1)) / st.dt
    compare(ob, sim, f"ch_grid = .false. ({case})")
    sim.close()
