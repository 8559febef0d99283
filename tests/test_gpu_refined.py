"""Refined (multi-level) domains on the GPU against the oracle's multi-level
driver (oracle/amr.py), bit for bit: the guard cells after the first
boundary update (same-level copies and prolongation from the coarser level),
and every block's state and the time state after whole steps (finest level
first, fine->coarse flux correction, leaf-cell CFL)."""
import numpy as np
import pytest

import amr
from helpers import assert_bitexact, setup_for
from piernik_b200 import problems
from piernik_b200.sim import Simulation

pytestmark = pytest.mark.gpu

DOM3 = (16, 16, 16)
REG3 = [((8, 8, 8), (24, 24, 24)), ((24, 24, 24), (40, 40, 40))]
DOM2 = (16, 16, 1)
REG2 = [((8, 6, 0), (24, 22, 1)), ((22, 18, 0), (38, 34, 1))]


def case(phys, dom, regions, lim="vanleer", fluids=None, fields=None, **kw):
    layout = problems.refined_layout(dom, regions, sizes=(8, 16), seed=3)
    setup = setup_for(phys, n=tuple(8 if d > 1 else 1 for d in dom), lim=lim, **kw)
    if fluids is not None:
        setup = setup.replace(fluids=fluids)
    return problems.refined_blocks(dom, layout, setup, fields or problems.wave_fields(dom, seed=5))


def library(dom, blocks, graph=False):
    sim = Simulation(blocks[0][0])
    for s, *_ in blocks[1:]:
        sim.add_block(s)
    sim.set_domain(dom, (True, True, True))
    for i, (s, L, off, u, b, psi) in enumerate(blocks):
        sim.place_block(i, off, L)
        sim.upload(u, b, psi, block=i)
    sim.update_boundaries()
    if graph:
        sim.use_graph(True)
    return sim


def compare(sim, a, what):
    for i, ob in enumerate(a.blocks):
        u, b, psi = sim.download(block=i)
        assert_bitexact(u, ob.u, f"{what}: u of block {i} (level {a.level[i]})")
        if a.mag:
            assert_bitexact(b, ob.b, f"{what}: b of block {i}")
            assert_bitexact(psi, ob.psi, f"{what}: psi of block {i}")


CASES = {
    "hd-3d": dict(phys="hd", dom=DOM3, regions=REG3),
    "mhd-3d-moncen": dict(phys="mhd", dom=DOM3, regions=REG3, lim="moncen"),
    "mhd-2d": dict(phys="mhd", dom=DOM2, regions=REG2),
    "mhd-3d-weno3": dict(phys="mhd", dom=DOM3, regions=REG3, lim="weno3"),
}


@pytest.mark.parametrize("phys", ["hd", "mhd"])
def test_refined_single_sweeps(gpu_lib, phys):
    """One sweep along each direction at a fixed dt, compared after each."""
    blocks = case(phys, DOM3, REG3)
    a = amr.AmrOracle(DOM3, blocks)
    a.fill_guards()
    sim = library(DOM3, blocks)
    for d in range(3):
        a.sweep(d, 0.004, 1.5)
        sim.sweep(d + 1, 0.004, 1.5)
        compare(sim, a, f"after the sweep along {'xyz'[d]}")
    sim.close()


@pytest.mark.parametrize("name", sorted(CASES) + ["mhd-3d-moncen+graph", "hd-3d+v1", "mhd-3d-moncen+v2", "mhd-3d-moncen+v3"])
def test_refined_matches_oracle(gpu_lib, name):
    graph = name.endswith("+graph")
    c = CASES[name.split("+")[0]]
    blocks = case(**c)
    a = amr.AmrOracle(c["dom"], blocks)
    a.fill_guards()
    sim = library(c["dom"], blocks, graph=graph)
    if "+v" in name:
        sim.set_stage_variant(int(name[-1]))               # another launch shape, the same arithmetic
    compare(sim, a, "after the first boundary update")
    a.run(3)
    sim.run(3)
    compare(sim, a, "after 3 steps")
    st = sim.time_state
    assert (st.t, st.dt, st.nstep) == (a.state.t, a.state.dt, a.state.nstep)
    sim.close()


@pytest.mark.parametrize("name", ["mhd-3d-moncen", "hd-3d", "mhd-2d", "mhd-3d-moncen+graph"])
def test_refined_one_launch_equals_per_level(gpu_lib, name):
    """The one-launch refined stage (every level's tiles and the flux
    restriction between them in one persistent work list, pk_set_refined_launch)
    against the default level-by-level launches: 3 steps, every block bit for
    bit, guard cells included, and no bounded wait gave up."""
    from piernik_b200._lib import PK_ST_TIMEOUT
    graph = name.endswith("+graph")
    c = CASES[name.split("+")[0]]
    blocks = case(**c)
    out = []
    for one in (False, True):
        sim = library(c["dom"], blocks, graph=graph)
        sim.set_refined_launch(one)
        sim.run(3)
        assert not sim.status() & PK_ST_TIMEOUT
        out.append([sim.download(block=i) for i in range(len(blocks))])
        sim.close()
    for i, (ref, got) in enumerate(zip(*out)):
        for k, (x, y) in enumerate(zip(ref, got)):
            if x is not None:
                assert_bitexact(y, x, f"{name}: array {k} of block {i}")


def test_refined_three_fluids_blast(gpu_lib):
    """Ion MHD + neutral + dust with an off-centre blast across all levels."""
    fl = [("ion", 5.0 / 3.0), ("neu", 1.4), ("dst", -1.0)]
    blocks = case("mhd", DOM3, REG3, fluids=fl, smalld=1.0e-4,
                  fields=problems.blast_fields(centre=(13.0, 12.0, 12.5), radius=2.5))
    a = amr.AmrOracle(DOM3, blocks)
    a.fill_guards()
    sim = library(DOM3, blocks)
    a.run(3)
    sim.run(3)
    compare(sim, a, "3-fluid blast after 3 steps")
    sim.close()


def test_refined_conserves_on_gpu(gpu_lib):
    """Leaf totals of the library's state are conserved to round-off."""
    blocks = case("mhd", DOM3, REG3)
    a = amr.AmrOracle(DOM3, blocks)
    a.fill_guards()
    t0 = amr.leaf_totals(a)
    scale = amr.leaf_totals(a, absolute=True)
    sim = library(DOM3, blocks)
    sim.run(4)
    for i, ob in enumerate(a.blocks):
        ob.u[...], ob.b[...], ob.psi[...] = sim.download(block=i)
    assert np.all(np.abs(amr.leaf_totals(a) - t0) <= 1e-12 * scale)
    sim.close()


@pytest.mark.parametrize("dom,reg", [(DOM3, REG3), (DOM2, REG2)])
def test_refined_restriction_matches_oracle(gpu_lib, dom, reg):
    blocks = case("mhd", dom, reg)
    a = amr.AmrOracle(dom, blocks)
    a.fill_guards()
    sim = library(dom, blocks)
    a.run(2)
    sim.run(2)
    a.restrict()
    sim.restrict()
    compare(sim, a, "after restriction")
    sim.close()


@pytest.mark.parametrize("orders,nb", [((0, -2), 4), ((0, 3), 4), ((1, 4), 4), ((0, -3), 4), ((1, -4), 4),
                                        ((0, 5), 6), ((1, -5), 6), ((0, 6), 6), ((0, -6), 6), ((1, 1), 4)])
def test_refined_prolongation_orders(gpu_lib, orders, nb):
    """Every prolongation order of the reference (ord_fluid_prolong,
    ord_mag_prolong; stencil ranges up to 3 need nb = 6), bit for bit."""
    blocks = case("mhd", DOM3, REG3, nb=nb, ord_fluid_prolong=orders[0], ord_mag_prolong=orders[1])
    a = amr.AmrOracle(DOM3, blocks)
    a.fill_guards()
    sim = library(DOM3, blocks)
    compare(sim, a, "after the first boundary update")
    a.run(2)
    sim.run(2)
    compare(sim, a, "after 2 steps")
    sim.close()


@pytest.mark.parametrize("phys,dom,reg,lim", [("hd", DOM3, REG3, "vanleer"), ("mhd", DOM3, REG3, "moncen"),
                                              ("mhd", DOM2, REG2, "vanleer"), ("mhd", DOM3, REG3, "weno3")])
def test_refined_unsplit_matches_oracle(gpu_lib, phys, dom, reg, lim):
    """The unsplit scheme on a refined domain: per stage every level's face
    fluxes finest first with the fine/coarse flux replacement, their
    application, then the guard update of uh (first stage) or u."""
    blocks = case(phys, dom, reg, lim=lim, solver="unsplit", cfl=0.3, cfl_glm=0.3)
    a = amr.AmrOracle(dom, blocks)
    a.fill_guards()
    sim = library(dom, blocks)
    a.run(3)
    sim.run(3)
    compare(sim, a, "unsplit, 3 steps")
    st = sim.time_state
    assert (st.t, st.dt, st.nstep) == (a.state.t, a.state.dt, a.state.nstep)
    sim.close()
