"""Parity at the benchmarked configurations, at full size.

The other parity tests compare small blocks; these run the configurations the
benchmark times, with the kernel instances and tile shapes the benchmark
uses, against the oracle (the reference's main loop fluidupdate.F90:99-136,
every pencil through solve_cg_riemann.F90:318-376):

* the 64^3 Sedov blast (HLLC, van Leer, CFL 0.7), 50 main-loop steps;
* the 256^3 MHD turbulence block (HLLD + GLM, moncen, CFL 0.5) for 2 steps
  with the tiles the autotuner picks at 256^3 (x: one whole 256-cell pencil
  per 256-thread CTA; y, z: 7 pencils x (64 + 8) cells in 512-thread CTAs);
* the same recipe at 128^3 for 100 steps, where besides bit equality the
  state must agree with the oracle's to 1e-9 relative (per component plane,
  max |a - b| over max |b|) -- the bound the path is specified with;
* the refined-blast layout of the uneven-blocks workload (515 blocks on three
  levels, ion MHD + neutral + dust), one step through a CUDA graph;
* the 512^2 Orszag-Tang vortex of the differentiable workload, 2 steps, and
  its adjoint over one step against the tangent-linear oracle.
"""
import numpy as np
import pytest

import amr
import oracle
from helpers import assert_bitexact, to_soa
from piernik_b200 import problems
from piernik_b200.sim import Simulation

pytestmark = pytest.mark.gpu

# tiles of the benchmark's 256^3 run: (pencils, owned cells, launch-bound variant)
BENCH_TILES_256 = {0: (1, 256, 2), 1: (7, 64, 6), 2: (7, 64, 6)}
BENCH_TILES_128 = {0: (1, 128, 2), 1: (7, 64, 6), 2: (7, 64, 6)}
REL_100 = 1.0e-9


def plane_rel(a, b):
    """max over component planes of max|a - b| / max|b|.  a, b: u or B in
    the reference's layout ([k, j, i, v]) or psi ([k, j, i], one plane)."""
    a, b = np.asarray(a), np.asarray(b)
    if a.ndim == 3:
        a, b = a[..., None], b[..., None]
    a, b = a.reshape(-1, a.shape[-1]), b.reshape(-1, b.shape[-1])
    scale = np.maximum(np.abs(b).max(axis=0), 1e-300)
    return float((np.abs(a - b).max(axis=0) / scale).max())


def run_both(setup, u, b, psi, nsteps, tiles=None):
    sim = Simulation(setup)
    sim.upload(u, b, psi)
    if tiles:
        for d, (P, L, V) in tiles.items():
            sim.set_tile(d, P, L, V)
    sim.run(nsteps)
    ob = oracle.OracleBlock(setup, u, b, psi)
    ob.run(nsteps)
    return sim, ob


def check_same(sim, ob, what):
    gu, gb, gp = sim.download()
    assert_bitexact(gu, ob.u, what + " u")
    if ob.setup.magnetic:
        assert_bitexact(gb, ob.b, what + " b")
        assert_bitexact(gp, ob.psi, what + " psi")
    st = sim.time_state
    assert (st.t, st.dt, st.nstep) == (ob.state.t, ob.state.dt, ob.state.nstep), what


def test_sedov_64_50_steps(gpu_lib, oracle_lib):
    """The 3D Sedov blast at the benchmarked size: 64^3, HLLC + van Leer, CFL 0.7, 50 steps."""
    setup, u, b, psi = problems.sedov(n=64)
    sim, ob = run_both(setup, u, b, psi, 50)
    check_same(sim, ob, "sedov 64^3 x 50")
    sim.close()


def test_mhd_turbulence_256_bench_tiles(gpu_lib, oracle_lib):
    """The headline block, 256^3 MHD, with the benchmark's tile shapes: the
    x sweep's whole 256-cell circular pencil and the 512-thread y/z tiles."""
    setup, u, b, psi = problems.mhd_turbulence(n=256, seed=1)
    sim, ob = run_both(setup, u, b, psi, 2, BENCH_TILES_256)
    check_same(sim, ob, "mhd 256^3 x 2")
    sim.close()


def test_mhd_turbulence_256_staged_tiles(gpu_lib, oracle_lib):
    """The headline block with the TMA-staged whole-pencil kernel along y and z."""
    from piernik_b200._lib import PK_VARIANT_STAGED
    setup, u, b, psi = problems.mhd_turbulence(n=256, seed=1)
    tiles = {0: (1, 256, 2), 1: (2, 256, PK_VARIANT_STAGED), 2: (2, 256, PK_VARIANT_STAGED)}
    sim, ob = run_both(setup, u, b, psi, 2, tiles)
    check_same(sim, ob, "mhd 256^3 x 2, staged y/z")
    sim.close()


def test_mhd_turbulence_128_100_steps(gpu_lib, oracle_lib):
    """100 main-loop steps (200 time steps) of the turbulence recipe at 128^3:
    bit for bit, and so within the 1e-9 relative bound after 100 steps."""
    setup, u, b, psi = problems.mhd_turbulence(n=128, seed=2)
    sim, ob = run_both(setup, u, b, psi, 100, BENCH_TILES_128)
    gu, gb, gp = sim.download()
    rel = max(plane_rel(gu, ob.u), plane_rel(gb, ob.b), plane_rel(gp, ob.psi))
    assert rel <= REL_100, f"relative difference {rel:.3e} after 100 steps"
    check_same(sim, ob, "mhd 128^3 x 100")
    sim.close()


def test_refined_blast_layout_one_step(gpu_lib, oracle_lib):
    """The uneven-blocks workload's layout (515 blocks on three levels, edges
    16..64, ion MHD + neutral + dust) for one step through a CUDA graph, as
    the benchmark runs it."""
    dom, blocks = problems.refined_blast()
    assert len(blocks) == 515
    a = amr.AmrOracle(dom, blocks)
    a.fill_guards()
    sim = Simulation(blocks[0][0])
    for s, *_ in blocks[1:]:
        sim.add_block(s)
    sim.set_domain(dom, (True, True, True))
    for i, (s, L, off, u, b, psi) in enumerate(blocks):
        sim.place_block(i, off, L)
        sim.upload(u, b, psi, block=i)
    sim.update_boundaries()
    sim.use_graph(True)
    a.run(1)
    sim.run(1)
    for i, ob in enumerate(a.blocks):
        gu, gb, gp = sim.download(block=i)
        assert_bitexact(gu, ob.u, f"u of block {i} (level {a.level[i]})")
        assert_bitexact(gb, ob.b, f"b of block {i}")
        assert_bitexact(gp, ob.psi, f"psi of block {i}")
    st = sim.time_state
    assert (st.t, st.dt, st.nstep) == (a.state.t, a.state.dt, a.state.nstep)
    sim.close()


def test_orszag_tang_512_forward_and_adjoint(gpu_lib, oracle_lib):
    """The differentiable workload's 512^2 Orszag-Tang vortex: 2 forward steps
    bit for bit, then the adjoint of one step against the tangent-linear
    oracle along two density-perturbation directions (to 1e-10)."""
    from test_gpu_adjoint import _tangent_dot, grad_at, interior_mask, put

    s, u, b, psi = problems.orszag_tang(n=512, seed=1)
    sim, ob = run_both(s, u, b, psi, 2)
    check_same(sim, ob, "orszag-tang 512^2 x 2")
    x0 = to_soa(s, u, b, psi)
    put(sim, x0)
    sim.time_state = type(sim.time_state)()
    dts = sim.grad_forward(1, 1)
    m = interior_mask(s, sim.nplanes)
    gd = s.guards
    rng = np.random.default_rng(7)
    for k in range(2):
        v = np.zeros_like(x0)
        v[0, :, gd[1]:gd[1] + 512, gd[0]:gd[0] + 512] = problems.gaussian_random_field((512, 512), 8.0, rng)
        w = np.where(m, rng.standard_normal(m.shape), 0.0)
        g, _ = grad_at(sim, x0, w, 1, 1, dts)
        ad = float(np.sum(g * v))
        tg, scale = _tangent_dot(s, x0, v, w, dts)
        rel = abs(ad - tg) / max(abs(tg), scale, 1e-300)
        assert rel <= 1e-10, f"direction {k}: adjoint {ad!r} vs tangent {tg!r} (rel {rel:.2e})"
    sim.close()
