"""E-GLM sources (hdc.F90:355-457, ``use_eglm``) on the GPU against the
oracle, bit for bit: after each triple of sweeps the guard cells are
refreshed, divB and grad(psi) are taken from the neighbours, the ionized
fluid's momentum, field, energy and psi get the sources in the reference's
statement order, the guards are refreshed again and psi is damped."""
import numpy as np
import pytest

import oracle
from helpers import assert_bitexact, random_state, setup_for
from piernik_b200 import problems
from piernik_b200._lib import PK_VARIANT_STAGED, PkError
from piernik_b200.sim import Simulation

pytestmark = pytest.mark.gpu


def _case(name):
    if name.startswith("turbulence"):
        s, u, b, psi = problems.mhd_turbulence(n=20, seed=3)
        return s.replace(use_eglm=True), u, b, psi, 5
    if name == "orszag-tang-2d":
        s, u, b, psi = problems.orszag_tang(n=32, seed=1)
        return s.replace(use_eglm=True), u, b, psi, 5
    s = setup_for("mhd", n=(20, 16, 12), lim="moncen").replace(fluids=[("ion", 5.0 / 3.0), ("neu", 1.4)],
                                                               use_eglm=True)
    u, b, psi = random_state(s, seed=8)
    return s, u, b, psi, 3


@pytest.mark.parametrize("name", ["turbulence", "turbulence+graph", "turbulence+staged", "orszag-tang-2d",
                                  "ion+neutral-random"])
def test_eglm_run_bitexact(gpu_lib, oracle_lib, name):
    s, u, b, psi, nsteps = _case(name)
    ob = oracle.OracleBlock(s, u, b, psi)
    sim = Simulation(s)
    sim.upload(u, b, psi)
    if name.endswith("+graph"):
        sim.use_graph(True)
    if name.endswith("+staged"):
        for d in range(3):
            sim.set_tile(d, 2, 0, PK_VARIANT_STAGED)
    ob.run(nsteps)
    sim.run(nsteps)
    st = sim.time_state
    assert st.t == ob.state.t and st.dt == ob.state.dt and st.nstep == ob.state.nstep
    gu, gb, gp = sim.download()
    assert_bitexact(gu, ob.u, f"{name} u")
    assert_bitexact(gb, ob.b, f"{name} b")
    assert_bitexact(gp, ob.psi, f"{name} psi")
    sim.close()


def test_eglm_changes_the_solution(gpu_lib):
    """The sources are really applied: the same run without them differs."""
    s, u, b, psi, _ = _case("turbulence")
    out = []
    for on in (False, True):
        sim = Simulation(s.replace(use_eglm=on))
        sim.upload(u, b, psi)
        sim.run(2)
        out.append(sim.download()[0])
        sim.close()
    assert not np.array_equal(out[0], out[1])


def test_eglm_slabs_equal_one_block(gpu_lib):
    """Two z-slabs of a connected domain: E-GLM's guard refreshes cross ranks
    (the halo callback), and the result equals one block's bit for bit."""
    from test_gpu_slabs import exact, run_ranks
    full = exact(setup_for("mhd", n=(24, 30, 32), lim="moncen")).replace(use_eglm=True)
    state = random_state(full, seed=9)
    one = Simulation(full)
    one.upload(*state)
    one.run(3)
    ref = one.download()
    one.close()
    g = full.guards
    for (n, off), arrs, _, _ in run_ranks(full, state, 2, 3, 2):
        for k in range(3):
            mine = arrs[k][g[2]:g[2] + n[2], g[1]:g[1] + n[1], g[0]:g[0] + n[0]]
            want = ref[k][tuple(slice(g[d] + off[d], g[d] + off[d] + n[d]) for d in (2, 1, 0))]
            assert_bitexact(mine, want, f"eglm slab {off} array {k}")


def test_eglm_rejections(gpu_lib):
    """The reference stops when E-GLM meets the unsplit scheme (hdc.F90:388);
    the differentiable path has no E-GLM sources."""
    s, u, b, psi, _ = _case("turbulence")
    with pytest.raises(Exception):
        Simulation(s.replace(solver="unsplit"))
    sim = Simulation(s)
    sim.upload(u, b, psi)
    with pytest.raises(PkError, match="E-GLM"):
        sim.grad_forward(1, 1)
    sim.close()
