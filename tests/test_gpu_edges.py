"""Edge geometries of the sweep path against the oracle, bit for bit: 1D
runs along each axis, 2D runs in the xz and yz planes, the smallest periodic
block (n = nb = 4 per axis), blocks thinner than the guard depth in one
direction, pencils longer than any CTA (halo tiles on the fused path), and
two fluids with WENO3."""
import pytest

import oracle
from helpers import assert_bitexact, random_state, setup_for, smooth_state
from piernik_b200.sim import Simulation

pytestmark = pytest.mark.gpu


def run_both(s, nsteps, seed=0, smooth=False):
    u, b, psi = (smooth_state if smooth else random_state)(s, seed=seed)
    ob = oracle.OracleBlock(s, u, b, psi)
    ob.fill_guards()
    sim = Simulation(s)
    sim.upload(ob.u, ob.b, ob.psi)
    assert ob.run(nsteps) == 0
    sim.run(nsteps)
    gu, gb, gp = sim.download()
    assert_bitexact(gu, ob.u, "u")
    if s.magnetic:
        assert_bitexact(gb, ob.b, "b")
        assert_bitexact(gp, ob.psi, "psi")
    st = sim.time_state
    assert (st.t, st.dt, st.nstep) == (ob.state.t, ob.state.dt, ob.state.nstep)
    sim.close()


@pytest.mark.parametrize("phys", ["hd", "mhd"])
@pytest.mark.parametrize("n", [(64, 1, 1), (1, 48, 1), (1, 1, 40), (24, 1, 20), (1, 18, 22)])
@pytest.mark.parametrize("solver", ["split", "unsplit"])
def test_lower_dimensional_runs(gpu_lib, oracle_lib, phys, n, solver):
    kw = {"cfl": 0.3, "cfl_glm": 0.3} if solver == "unsplit" else {}
    run_both(setup_for(phys, n=n, lim="moncen", solver=solver, **kw), 4, seed=2)


@pytest.mark.parametrize("n", [(4, 4, 4), (5, 4, 7), (4, 9, 4)])
def test_smallest_periodic_blocks(gpu_lib, oracle_lib, n):
    run_both(setup_for("mhd", n=n, lim="vanleer"), 3, seed=4, smooth=True)


@pytest.mark.parametrize("n", [(600, 4, 4), (4, 530, 4)])
def test_pencils_longer_than_a_cta(gpu_lib, oracle_lib, n):
    run_both(setup_for("mhd", n=n, lim="minmod"), 2, seed=6, smooth=True)


def test_two_fluids_weno3(gpu_lib, oracle_lib):
    """Ion MHD + neutral through WENO3 (a moving dust fluid under HLLD can
    reach the reference's 0/0 at diverging faces, whose NaN bit patterns
    differ between host and device)."""
    s = setup_for("mhd", n=(12, 10, 8), lim="weno3").replace(fluids=[("ion", 5.0 / 3.0), ("neu", 1.4)])
    run_both(s, 3, seed=1, smooth=True)


@pytest.mark.parametrize("n", [(8, 100, 6), (6, 8, 90)])
def test_stage_path_chunked_y_z(gpu_lib, oracle_lib, n):
    """Outflow boundaries take the stage path; y and z pencils longer than 80
    cells run there in chunks with a 2-cell halo (fewer than four whole
    pencils would fit a CTA)."""
    from piernik_b200.config import BND_OUT
    s = setup_for("hd", n=n, lim="moncen").replace(bnd=((BND_OUT, BND_OUT),) * 3)
    run_both(s, 2, seed=8, smooth=True)
