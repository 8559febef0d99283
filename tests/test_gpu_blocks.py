"""Connected blocks of one level on one device (guard exchange between
blocks, cg_list_bnd.F90:251-324, after every RK stage as sweeps.F90:217-272
does): a domain tiled by blocks of uneven sizes must evolve exactly like the
same domain held as one block, because every interior cell sees the same
neighbours through the guard cells.  The single block runs the fused sweep,
which the oracle parity tests pin bit for bit."""
import numpy as np
import pytest

from helpers import assert_bitexact, random_state, setup_for
from piernik_b200.config import BND_OUT, BND_PER
from piernik_b200.sim import Simulation

pytestmark = pytest.mark.gpu


def tiles(xs, ys, zs):
    out = []
    oz = 0
    for bz in zs:
        oy = 0
        for by in ys:
            ox = 0
            for bx in xs:
                out.append(((bx, by, bz), (ox, oy, oz)))
                ox += bx
            oy += by
        oz += bz
    return out


def window(setup, arr, n, off):
    if arr is None:
        return None
    g = setup.guards
    sl = tuple(slice(off[d], off[d] + n[d] + 2 * g[d]) for d in (2, 1, 0))
    return np.ascontiguousarray(arr[sl])


def interior_of(setup, arr, n, off):
    g = setup.guards
    return arr[tuple(slice(g[d] + off[d], g[d] + off[d] + n[d]) for d in (2, 1, 0))]


def exact_dl(setup):
    """Cell size 1/8 (exact in binary), so that every block's (xmax - xmin)/n
    equals the level's dl bit for bit."""
    return setup.replace(xmin=(0.0, 0.0, 0.0), xmax=tuple(0.125 * setup.n[d] for d in range(3)))


def run_tiled(full, state, blocks, periodic, nsteps, bnd_x=BND_PER, graph=False):
    u, b, psi = state
    sims = None
    for i, (n, off) in enumerate(blocks):
        bnd = list(full.bnd)
        if not periodic[0]:
            lo = bnd_x if off[0] == 0 else BND_PER
            hi = bnd_x if off[0] + n[0] == full.n[0] else BND_PER
            bnd[0] = (lo, hi)
        s = full.replace(n=n, bnd=tuple(bnd),
                         xmin=tuple(full.xmin[d] + off[d] * full.dl[d] for d in range(3)),
                         xmax=tuple(full.xmin[d] + (off[d] + n[d]) * full.dl[d] for d in range(3)))
        if sims is None:
            sims = Simulation(s)
            sims.set_domain(full.n, periodic)
            bid = 0
        else:
            bid = sims.add_block(s)
        sims.place_block(bid, off)
        sims.upload(window(full, u, n, off), window(full, b, n, off), window(full, psi, n, off), block=bid)
    sims.update_boundaries()
    if graph:
        sims.use_graph(True)
    sims.run(nsteps)
    out = []
    for i, (n, off) in enumerate(blocks):
        out.append(sims.download(block=i))
    st = sims.time_state
    sims.close()
    return out, st


@pytest.mark.parametrize("phys,graph", [("hd", False), ("mhd", False), ("mhd", True)])
def test_tiled_periodic_domain_equals_one_block(gpu_lib, phys, graph):
    """A periodic domain tiled completely: exchange before each sweep, then the
    batched fused sweep reading its halo from the guards."""
    full = exact_dl(setup_for(phys, n=(40, 36, 28), lim="moncen"))
    state = random_state(full, seed=3)
    one = Simulation(full)
    one.upload(*state)
    one.run(3)
    ref = one.download()
    st1 = one.time_state
    one.close()
    blocks = tiles([16, 24], [20, 16], [12, 16])
    got, st2 = run_tiled(full, state, blocks, (True, True, True), 3, graph=graph)
    assert st1.t == st2.t and st1.dt == st2.dt
    for (n, off), arrs in zip(blocks, got):
        s = full.replace(n=n)
        for k, name in enumerate(("u", "b", "psi")):
            if arrs[k] is None:
                continue
            assert_bitexact(interior_of(s, arrs[k], n, (0, 0, 0)), interior_of(full, ref[k], n, off),
                            f"{phys} block {off} {name}")


def test_tiled_outflow_domain_equals_one_block(gpu_lib):
    """Outflow along x: the per-stage path (pk_solve_cg per block, then the
    blocks' own outflow rule and the exchange after each stage)."""
    full = exact_dl(setup_for("hd", n=(40, 20, 16), lim="vanleer", bnd=((BND_OUT, BND_OUT), (BND_PER, BND_PER),
                                                                       (BND_PER, BND_PER))))
    state = random_state(full, seed=4)
    one = Simulation(full)
    one.upload(*state)
    one.update_boundaries()          # the recipe's guards are periodic images; start both from outflow ones
    one.run(3)
    ref = one.download()
    one.close()
    blocks = tiles([12, 16, 12], [20], [8, 8])
    got, _ = run_tiled(full, state, blocks, (False, True, True), 3, bnd_x=BND_OUT)
    for (n, off), arrs in zip(blocks, got):
        s = full.replace(n=n)
        assert_bitexact(interior_of(s, arrs[0], n, (0, 0, 0)), interior_of(full, ref[0], n, off), f"block {off}")


def test_tiled_domain_with_a_hole_uses_stages(gpu_lib):
    """Blocks that do not cover the periodic domain still exchange what they
    share; the run equals the same blocks swept one stage at a time."""
    full = exact_dl(setup_for("hd", n=(32, 16, 16), lim="vanleer"))
    state = random_state(full, seed=5)
    blocks = tiles([16, 16], [16], [16])[:1] + [((8, 16, 16), (16, 0, 0))]
    got, _ = run_tiled(full, state, blocks, (True, True, True), 2)
    assert all(np.isfinite(g[0]).all() for g in got)


def test_overlapping_blocks_are_rejected(gpu_lib):
    full = setup_for("hd", n=(16, 16, 16))
    s = full.replace(n=(8, 16, 16))
    sim = Simulation(s)
    sim.set_domain(full.n, (True, True, True))
    b1 = sim.add_block(s)
    sim.place_block(0, (0, 0, 0))
    sim.place_block(b1, (4, 0, 0))
    with pytest.raises(RuntimeError, match="overlap"):
        sim.update_boundaries()
    sim.close()
