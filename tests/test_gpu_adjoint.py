"""The differentiable path: adjoint sweep kernel and checkpointed backward
pass against central finite differences of the forward CUDA path.

Directional check: for random interior directions V and weights W,
<J^T W, V> must match (<W, F(X + eps V)> - <W, F(X - eps V)>) / (2 eps) with
eps = 1e-6 to a relative 1e-8, along 16 directions; F is one fused sweep or
K whole steps at a fixed dt sequence.  The error is relative to the larger of
|FD| and the l2 norm of the per-value terms w_i (F+ - F-)_i / (2 eps): a sum
of random-sign terms can cancel to far below its terms, and the rounding of
the finite difference scales with the terms, not with the sum.

The sweep is piecewise smooth: min/max of the two face states' wave speeds,
limiter switches and HLLD region tests are kinks, and a direction whose
+-eps segment crosses one has no central difference to compare with.  Such a
direction shows itself by a finite difference that changes with eps (eps and
eps/10 disagree beyond the tolerance); it is counted and replaced by a fresh
draw.  A direction whose finite difference is stable must match.

Over several steps nearly every full-grid direction crosses some kink (tens
of thousands of face evaluations), so the multi-step checks perturb one cell
(all its variables) at a time; the rounding of such a small derivative's
finite difference is near 1e-8 of it, so their tolerance is 1e-6.  The
moncen limiter switches between its centred and one-sided slopes wherever a
neighbour difference is three times the other, so on a 16 x 12 x 10 block a
full-grid direction almost always crosses one: its single-sweep check also
perturbs one cell at a time.  The Orszag-Tang check follows the workload's
definition: the loss is the central magnetic energy, the directions are
seeded Gaussian random fields of the relative density perturbation.
"""
import numpy as np
import pytest

from helpers import from_soa, random_state, setup_for, smooth_state, to_soa
from piernik_b200 import problems
from piernik_b200._lib import PK_LAYOUT_SOA, PK_ST_TIMEOUT
from piernik_b200.sim import Simulation

pytestmark = pytest.mark.gpu

EPS = 1.0e-6
RTOL = 1.0e-8
NDIR = 16
MAX_DRAWS = 64


def interior_mask(setup, nplanes):
    m = np.zeros((nplanes,) + tuple(setup.ext[::-1]), dtype=bool)
    g, n = setup.guards, setup.n
    m[:, g[2]:g[2] + n[2], g[1]:g[1] + n[1], g[0]:g[0] + n[0]] = True
    return m


def put(sim, x):
    u, b, psi = from_soa(sim.setup, x)
    sim.upload(np.ascontiguousarray(u), None if b is None else np.ascontiguousarray(b),
               None if psi is None else np.ascontiguousarray(psi), layout=PK_LAYOUT_SOA)


def get(sim):
    u, b, psi = sim.download(layout=PK_LAYOUT_SOA)
    planes = [u] + ([b, psi[None]] if sim.setup.magnetic else [])
    return np.concatenate(planes, 0)


def directions(setup, nplanes, seed, count=MAX_DRAWS, one_cell=False):
    rng = np.random.default_rng(seed)
    m = interior_mask(setup, nplanes)
    cells = np.argwhere(m[0])
    for _ in range(count):
        if one_cell:
            v = np.zeros(m.shape)
            v[(slice(None),) + tuple(cells[rng.integers(0, len(cells))])] = rng.standard_normal(nplanes)
        else:
            v = np.where(m, rng.standard_normal(m.shape), 0.0)
        w = np.where(m, rng.standard_normal(m.shape), 0.0)
        yield v, w


def central(fwd, x0, v, w, m, eps):
    """Central difference of <W, F> along V and the l2 scale of its terms."""
    terms = np.where(m, w * (fwd(x0 + eps * v) - fwd(x0 - eps * v)), 0.0) / (2 * eps)
    return float(np.sum(terms)), float(np.sqrt(np.sum(terms * terms)))


def directional_check(fwd, adj, x0, setup, nplanes, seed, what, rtol=RTOL, one_cell=False):
    """fwd(x) -> F(x); adj(x, w, k) -> J(x)^T w for draw k.  Passes when NDIR
    directions with a stable finite difference all match."""
    m = interior_mask(setup, nplanes)
    clean = kinks = 0
    worst = 0.0
    for k, (v, w) in enumerate(directions(setup, nplanes, seed, one_cell=one_cell)):
        ad = float(np.sum(adj(x0, w, k) * v))
        fd, scale = central(fwd, x0, v, w, m, EPS)
        rel = abs(ad - fd) / max(abs(fd), scale, 1e-300)
        if rel > rtol:
            fd2, scale2 = central(fwd, x0, v, w, m, EPS / 10)
            if abs(fd - fd2) > rtol * max(abs(fd), scale, scale2):
                kinks += 1
                continue
            raise AssertionError(f"{what} direction {k}: adjoint {ad!r} vs finite difference {fd!r} "
                                 f"(rel {rel:.2e}, eps/10 gives {fd2!r})")
        worst = max(worst, rel)
        clean += 1
        if clean == NDIR:
            break
    assert clean == NDIR, f"{what}: only {clean} directions with a stable finite difference ({kinks} crossed kinks)"
    return worst, kinks


@pytest.mark.parametrize("phys,lim", [("hd", "vanleer"), ("hd", "minmod"), ("mhd", "vanleer"), ("mhd", "moncen")])
def test_adjoint_sweep_vs_fd(gpu_lib, phys, lim):
    s = setup_for(phys, n=(16, 12, 10), lim=lim)
    x0 = to_soa(s, *smooth_state(s, seed=2))
    sim = Simulation(s)
    dt, ch = 0.004, 1.1
    for cdim in (1, 2, 3):
        def fwd(x):
            put(sim, x)
            sim.sweep(cdim, dt, ch)
            return get(sim)

        def adj(x, w, k):
            put(sim, x)
            sim.adjoint_set(w)
            sim.adjoint_sweep(cdim, dt, ch)
            return sim.adjoint_get()

        directional_check(fwd, adj, x0, s, sim.nplanes, 7 + cdim, f"{phys}/{lim} sweep {cdim}",
                          one_cell=(lim == "moncen"))
    sim.close()


def grad_at(sim, x0, w, nsteps, every, dts=None):
    put(sim, x0)
    sim.time_state = type(sim.time_state)()
    got = sim.grad_forward(nsteps, every, dts)
    sim.adjoint_set(w)
    sim.grad_backward()
    return sim.adjoint_get(), got


def final_state(sim, x0, nsteps, dts):
    put(sim, x0)
    sim.time_state = type(sim.time_state)()
    sim.grad_forward(nsteps, nsteps, dts)
    return get(sim)


def multistep_check(sim, x0, K, every, seed, what):
    put(sim, x0)
    sim.time_state = type(sim.time_state)()
    dts = sim.grad_forward(K, every)
    return directional_check(lambda x: final_state(sim, x, K, dts),
                             lambda x, w, k: grad_at(sim, x, w, K, every, dts)[0],
                             x0, sim.setup, sim.nplanes, seed, what, rtol=1.0e-6, one_cell=True)


@pytest.mark.parametrize("phys", ["hd", "mhd"])
def test_multistep_gradient_vs_fd(gpu_lib, phys):
    s = setup_for(phys, n=(12, 12, 12), lim="vanleer")
    x0 = to_soa(s, *smooth_state(s, seed=4))
    sim = Simulation(s)
    multistep_check(sim, x0, 4, 2, 9, f"{phys} 4 steps")
    sim.close()


def test_orszag_tang_gradient_vs_fd(gpu_lib):
    """The differentiable Orszag-Tang workload at 32^2: loss = magnetic energy
    of the central 8^2 cells after K = 6 steps, gradient with respect to the
    relative density perturbation field (1e-3 x a seeded unit-rms Gaussian
    random field at the base point) through torch.autograd (checkpoint every
    2 steps), against central differences along 16 seeded Gaussian random
    directions at the dt sequence of the unperturbed run.

    The vortex's velocity and field are uniform along one axis each, so after
    a density perturbation of 1e-3 the two face states of most faces differ by
    about 1e-3 of their size: min/max switches of the wave-speed estimates sit
    that close to the base point everywhere, and a central difference over
    +-eps crosses a share of them that grows with eps.  Its error therefore
    falls in proportion to eps (measured: about 1e-5 at eps = 1e-6, 1e-7 to
    1e-8 at eps = 1e-7); the check asks for that convergence and for
    agreement to 1e-6 of the directions' rms derivative at eps = 1e-7."""
    import torch
    from piernik_b200.autograd import advance, central_magnetic_energy, last_dts, orszag_tang_state

    n, K = 32, 6
    s = problems.orszag_tang_fields(n)[0]
    sim = Simulation(s)
    d0 = torch.tensor(1.0e-3 * problems.orszag_tang_perturbation(n, seed=1), device="cuda", requires_grad=True)
    out = advance(sim, orszag_tang_state(sim, d0), K, every=2)
    loss = central_magnetic_energy(sim, out)
    loss.backward()
    dts = last_dts(out)
    grad = d0.grad.detach().cpu().numpy()
    nv, cy = s.nvar, n // 4
    y0 = (n - cy) // 2
    dV = float(np.prod(s.dl))

    def central_b(d):
        with torch.no_grad():
            o = advance(sim, orszag_tang_state(sim, d), K, dts=dts)
            return o[nv:nv + 3, 0, y0:y0 + cy, y0:y0 + cy].cpu().numpy()

    def fd(vt, eps):
        # the loss difference summed cell by cell, (b+ - b-)(b+ + b-) / 2, so
        # that the sum of squares does not cancel
        bp, bm = central_b(d0.detach() + eps * vt), central_b(d0.detach() - eps * vt)
        return float(0.5 * ((bp - bm) * (bp + bm)).sum() * dV / (2 * eps))

    rng = np.random.default_rng(21)
    ads, err6, err7 = [], [], []
    for k in range(NDIR):
        v = problems.gaussian_random_field((n, n), 8.0, rng)
        vt = torch.tensor(v, device="cuda")
        ad = float(np.sum(grad * v))
        ads.append(ad)
        err6.append(abs(ad - fd(vt, EPS)))
        err7.append(abs(ad - fd(vt, EPS / 10)))
    rms = float(np.sqrt(np.mean(np.square(ads))))
    err6, err7 = np.array(err6) / rms, np.array(err7) / rms
    assert err7.max() <= 1.0e-6, f"eps=1e-7 errors {err7}"
    assert np.median(err7) < np.median(err6) / 3, f"no convergence in eps: {np.median(err6)} -> {np.median(err7)}"
    sim.close()


def test_checkpoint_interval_is_exact(gpu_lib):
    """Recomputing segments reproduces the forward bit for bit, so the gradient
    does not depend on the checkpoint interval."""
    s = setup_for("mhd", n=(12, 10, 8), lim="vanleer")
    x0 = to_soa(s, *smooth_state(s, seed=5))
    sim = Simulation(s)
    w = next(directions(s, sim.nplanes, seed=3, count=1))[1]
    K = 6
    put(sim, x0)
    dts = sim.grad_forward(K, 1)
    ref, _ = grad_at(sim, x0, w, K, 1, dts)
    for every in (2, 3, 4, 6, 7):
        g, _ = grad_at(sim, x0, w, K, every, dts)
        assert np.array_equal(g.view(np.uint64), ref.view(np.uint64)), f"every={every}"
    assert not np.any(ref[~interior_mask(s, sim.nplanes)]), "guard cells of the gradient are not zero"
    sim.close()


def test_recorded_forward_equals_run(gpu_lib):
    """pk_grad_forward without a dt sequence takes the same steps as pk_run."""
    s = setup_for("mhd", n=(12, 10, 8), lim="moncen")
    x0 = to_soa(s, *smooth_state(s, seed=6))
    a, b = Simulation(s), Simulation(s)
    put(a, x0)
    put(b, x0)
    dts = a.grad_forward(5, 2)
    b.run(5)
    assert np.array_equal(get(a).view(np.uint64), get(b).view(np.uint64))
    assert a.time_state.t == b.time_state.t and a.time_state.nstep == b.time_state.nstep == 5
    assert dts[0] > 0
    a.close()
    b.close()


def test_torch_autograd(gpu_lib):
    """advance() under torch.autograd gives the library's gradient."""
    import torch
    from piernik_b200.autograd import advance, last_dts

    s = setup_for("mhd", n=(12, 12, 8), lim="vanleer")
    x0 = to_soa(s, *smooth_state(s, seed=8))
    sim = Simulation(s)
    g, n = s.guards, s.n
    inner = (slice(None), slice(g[2], g[2] + n[2]), slice(g[1], g[1] + n[1]), slice(g[0], g[0] + n[0]))
    xi = torch.tensor(np.ascontiguousarray(x0[inner]), device="cuda", requires_grad=True)
    out = advance(sim, xi, 3, every=2)
    dts = last_dts(out)
    assert dts is not None and len(dts) == 3
    w = np.random.default_rng(1).standard_normal(tuple(out.shape))
    (out * torch.tensor(w, device="cuda")).sum().backward()
    grad = xi.grad.detach().cpu().numpy()
    # the same gradient through the C ABI directly
    wf = np.zeros_like(x0)
    wf[inner] = w
    ref, _ = grad_at(sim, x0, wf, 3, 2, dts)
    assert np.array_equal(grad.view(np.uint64), np.ascontiguousarray(ref[inner]).view(np.uint64))
    sim.close()


def test_adjoint_rejects_unsupported(gpu_lib):
    from piernik_b200.config import BND_OUT
    s = setup_for("hd", n=(8, 8, 8), bnd=((BND_OUT, BND_OUT),) * 3)
    sim = Simulation(s)
    put(sim, to_soa(s, *smooth_state(s)))
    with pytest.raises(RuntimeError, match="periodic"):
        sim.grad_forward(1, 1)
    sim.close()


def _tangent_dot(s, x0, v, w, dts):
    """<w, J v> from the tangent-linear oracle (CPU), interior cells."""
    import tangent
    m = interior_mask(s, s.nvar + (4 if s.magnetic else 0))
    u, b, psi = from_soa(s, x0)
    du, db, dp = from_soa(s, v)
    lay = lambda a: None if a is None else np.ascontiguousarray(np.moveaxis(a, 0, -1))
    (_, _, _), (tu, tb, tp) = tangent.jvp(s, lay(u), lay(b), None if psi is None else np.ascontiguousarray(psi),
                                          lay(du), lay(db), None if dp is None else np.ascontiguousarray(dp), dts)
    jv = to_soa(s, tu, tb, tp)
    terms = np.where(m, w * jv, 0.0)
    return float(terms.sum()), float(np.sqrt((terms * terms).sum()))


@pytest.mark.parametrize("phys,lim,n,K,state", [("hd", "vanleer", (12, 10, 8), 3, "random"),
                                                ("hd", "minmod", (16, 12, 10), 2, "smooth"),
                                                ("mhd", "moncen", (12, 10, 8), 3, "random"),
                                                ("mhd", "vanleer", (10, 10, 10), 4, "smooth")])
def test_adjoint_equals_tangent_oracle(gpu_lib, oracle_lib, phys, lim, n, K, state):
    """<J^T w, v> from the CUDA adjoint against <w, J v> from the CPU
    tangent-linear oracle along full-grid random directions: both
    differentiate the same branches (the primal values are bit-identical), so
    they agree to rounding even on noisy states where nearly every central
    difference crosses a kink."""
    s = setup_for(phys, n=n, lim=lim)
    x0 = to_soa(s, *(random_state(s, seed=12) if state == "random" else smooth_state(s, seed=12)))
    sim = Simulation(s)
    put(sim, x0)
    sim.time_state = type(sim.time_state)()
    dts = sim.grad_forward(K, 2)
    for k, (v, w) in enumerate(directions(s, sim.nplanes, seed=31, count=4)):
        g, _ = grad_at(sim, x0, w, K, 2, dts)
        ad = float(np.sum(g * v))
        tg, scale = _tangent_dot(s, x0, v, w, dts)
        rel = abs(ad - tg) / max(abs(tg), scale, 1e-300)
        assert rel <= 1e-10, f"{phys}/{lim} direction {k}: adjoint {ad!r} vs tangent {tg!r} (rel {rel:.2e})"
    sim.close()


def test_orszag_tang_adjoint_equals_tangent_oracle(gpu_lib, oracle_lib):
    """The Orszag-Tang vortex, whose central differences are kink-limited:
    adjoint against tangent along density-perturbation directions, 32^2, 6
    steps."""
    s, u, b, psi = problems.orszag_tang(n=32, seed=1)
    x0 = to_soa(s, u, b, psi)
    sim = Simulation(s)
    put(sim, x0)
    sim.time_state = type(sim.time_state)()
    dts = sim.grad_forward(6, 2)
    m = interior_mask(s, sim.nplanes)
    rng = np.random.default_rng(4)
    for k in range(3):
        v = np.zeros_like(x0)
        v[0] = np.where(m[0], rng.standard_normal(m[0].shape), 0.0)          # density only
        w = np.where(m, rng.standard_normal(m.shape), 0.0)
        g, _ = grad_at(sim, x0, w, 6, 2, dts)
        ad = float(np.sum(g * v))
        tg, scale = _tangent_dot(s, x0, v, w, dts)
        rel = abs(ad - tg) / max(abs(tg), scale, 1e-300)
        assert rel <= 1e-10, f"Orszag-Tang direction {k}: adjoint {ad!r} vs tangent {tg!r} (rel {rel:.2e})"
    sim.close()


@pytest.mark.parametrize("phys", ["hd", "mhd"])
def test_adjoint_tiles_agree(gpu_lib, phys):
    """Every launch-bound variant and owned length of the adjoint kernels
    (whole periodic pencils, chunks with a 3-cell halo, one or several
    pencils per CTA, and variant 5: the TMA-staged whole-pencil pair, which
    ignores the length) gives the same adjoint bit for bit, guard cells
    included: the arithmetic per cell does not depend on the tile.  The odd
    extent along y (35) leaves the last staged pencil pair with one pencil."""
    s = setup_for(phys, n=(40, 35, 34), lim="moncen")
    x0 = to_soa(s, *random_state(s, seed=5))
    sim = Simulation(s)
    rng = np.random.default_rng(9)
    w = np.where(interior_mask(s, sim.nplanes), rng.standard_normal(x0.shape), 0.0)
    dt, ch = 0.003, 1.2
    for cdim in (1, 2, 3):
        ref = None
        for variant in range(6):
            for length in (0, 7, 26, 40):
                sim.set_adjoint_tile(cdim - 1, length, variant)
                put(sim, x0)
                sim.adjoint_set(w)
                sim.adjoint_sweep(cdim, dt, ch)
                got = sim.adjoint_get()
                assert not sim.status() & PK_ST_TIMEOUT, f"{phys} sweep {cdim}: variant {variant} timed out"
                if ref is None:
                    ref = got
                else:
                    assert np.array_equal(got, ref), f"{phys} sweep {cdim}: variant {variant} length {length} differs"
    sim.set_adjoint_tile(-1, 0, -1)
    sim.close()


@pytest.mark.parametrize("phys", ["hd", "mhd"])
def test_staged_recording_sweep(gpu_lib, phys):
    """With the TMA-staged tile selected on every axis, the backward pass
    recomputes its segments with the staged kernel in recording mode (stage-1
    state and floor records from plain stores): the gradient equals the one
    recomputed with the default fused tiles bit for bit, and the recorded
    forward equals the plain forward."""
    from piernik_b200._lib import PK_VARIANT_STAGED
    s = setup_for(phys, n=(24, 20, 18), lim="moncen")
    x0 = to_soa(s, *random_state(s, seed=21))
    sim = Simulation(s)
    rng = np.random.default_rng(17)
    w = np.where(interior_mask(s, sim.nplanes), rng.standard_normal(x0.shape), 0.0)
    ref_g, ref_dts = grad_at(sim, x0, w, 4, 2)
    for d in range(3):
        sim.set_tile(d, 2, 0, PK_VARIANT_STAGED)
    got_g, got_dts = grad_at(sim, x0, w, 4, 2)
    assert np.array_equal(np.asarray(got_dts), np.asarray(ref_dts))
    assert np.array_equal(got_g, ref_g), f"{phys}: staged recording sweep changes the gradient"
    sim.close()
