"""Regridding a refined domain on the GPU against the oracle's multi-level
driver, bit for bit: refinement adds blocks on a finer level and fills
their interiors from the coarser one (pk_prolong_block, the refinement
update's prolongation); derefinement restricts and frees blocks
(pk_restrict, pk_block_remove, which moves the later block ids down); the
run carries on with the new couplings, leaf masks and time state."""
import numpy as np
import pytest

import amr
from helpers import assert_bitexact, setup_for
from piernik_b200 import problems
from piernik_b200.sim import Simulation

pytestmark = pytest.mark.gpu

DOM3 = (16, 16, 16)
REG1 = [((8, 8, 8), (24, 24, 24))]
NEW2 = [((24, 24, 24), (8, 8, 8)), ((32, 24, 24), (8, 8, 8))]


def case(phys, **kw):
    layout = problems.refined_layout(DOM3, REG1, sizes=(8, 16), seed=3)
    setup = setup_for(phys, n=(8, 8, 8), **kw)
    return problems.refined_blocks(DOM3, layout, setup, problems.wave_fields(DOM3, seed=5))


def new_blocks(blocks):
    made = problems.refined_blocks(DOM3, [(2, off, n) for off, n in NEW2], blocks[0][0],
                                   problems.wave_fields(DOM3, seed=5))
    return [(s, L, off) for s, L, off, *_ in made]


def compare(sim, a, what):
    for i, ob in enumerate(a.blocks):
        u, b, psi = sim.download(block=i)
        assert_bitexact(u, ob.u, f"{what}: u of block {i} (level {a.level[i]})")
        if a.mag:
            assert_bitexact(b, ob.b, f"{what}: b of block {i}")
            assert_bitexact(psi, ob.psi, f"{what}: psi of block {i}")


@pytest.mark.parametrize("phys,orders", [("hd", (0, 2)), ("mhd", (0, 2)), ("mhd", (1, -4)), ("mhd", (0, 4))])
def test_regrid_matches_oracle(gpu_lib, phys, orders):
    blocks = case(phys, ord_fluid_prolong=orders[0], ord_mag_prolong=orders[1])
    a = amr.AmrOracle(DOM3, blocks)
    a.fill_guards()
    sim = Simulation(blocks[0][0])
    for s, *_ in blocks[1:]:
        sim.add_block(s)
    sim.set_domain(DOM3, (True, True, True))
    for i, (s, L, off, u, b, psi) in enumerate(blocks):
        sim.place_block(i, off, L)
        sim.upload(u, b, psi, block=i)
    sim.update_boundaries()
    a.run(2)
    sim.run(2)
    compare(sim, a, "before refining")

    # refine: two level-2 blocks, filled from level 1
    add = new_blocks(blocks)
    a = a.relayout(add=add)
    a.fill_guards()
    ids = []
    for s, L, off in add:
        k = sim.add_block(s)
        sim.place_block(k, off, L)
        ids.append(k)
    sim.update_boundaries()
    for k in ids:
        a.prolong_block(k)
        sim.prolong_block(k)
    a.fill_guards()
    sim.update_boundaries()
    compare(sim, a, "after refining")
    a.run(2)
    sim.run(2)
    compare(sim, a, "2 steps after refining")
    st = sim.time_state
    assert (st.t, st.dt, st.nstep) == (a.state.t, a.state.dt, a.state.nstep)

    # derefine the first new block: restrict, free it (the second moves down one id)
    a.restrict()
    sim.restrict()
    compare(sim, a, "after restriction")
    a = a.relayout(remove=[ids[0]])
    a.fill_guards()
    sim.remove_block(ids[0])
    sim.update_boundaries()
    compare(sim, a, "after derefining")
    a.run(2)
    sim.run(2)
    compare(sim, a, "2 steps after derefining")
    st = sim.time_state
    assert (st.t, st.dt, st.nstep) == (a.state.t, a.state.dt, a.state.nstep)
    sim.close()


def test_prolong_block_rejects(gpu_lib):
    blocks = case("hd")
    sim = Simulation(blocks[0][0])
    for s, *_ in blocks[1:]:
        sim.add_block(s)
    sim.set_domain(DOM3, (True, True, True))
    for i, (s, L, off, u, b, psi) in enumerate(blocks):
        sim.place_block(i, off, L)
        sim.upload(u, b, psi, block=i)
    with pytest.raises(Exception, match="refined level"):
        sim.prolong_block(0)
    with pytest.raises(Exception):
        sim.remove_block(len(blocks))
    sim.close()
