"""Shared helpers of the test-suite: one state, two engines (oracle and CUDA)."""
import numpy as np

from piernik_b200.config import Setup
from piernik_b200 import problems


def setup_for(phys: str, n=(12, 10, 8), lim="vanleer", limb=None, bnd=None, **kw) -> Setup:
    """lim = 'weno3' selects interpol_str = 'weno3' (the limiters then play no part)."""
    mag = phys == "mhd"
    if lim == "weno3":
        kw.setdefault("interpolation", "weno3")
        lim = "vanleer"
    if limb == "weno3":
        limb = None
    s = Setup(n=tuple(n), fluids=[("ion", 5.0 / 3.0)] if mag else [("neu", 1.4)], magnetic=mag,
              limiter=lim, limiter_b=limb or lim, xmin=(0.0, 0.0, 0.0),
              xmax=(n[0] * 0.1, n[1] * 0.1, n[2] * 0.1), **kw)
    if bnd is not None:
        s = s.replace(bnd=bnd)
    return s


def interior(setup: Setup, a):
    g, n = setup.guards, setup.n
    return a[g[2]:g[2] + n[2], g[1]:g[1] + n[1], g[0]:g[0] + n[0]]


def assert_bitexact(a, b, what=""):
    a = np.asarray(a)
    b = np.asarray(b)
    assert a.shape == b.shape, (what, a.shape, b.shape)
    same = (a.view(np.uint64) == b.view(np.uint64))
    if not same.all():
        idx = np.argwhere(~same)
        i = tuple(idx[0])
        rel = np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300))
        raise AssertionError(f"{what}: {(~same).sum()} of {same.size} values differ; first at {i}: "
                             f"{a[i]!r} vs {b[i]!r}; max rel {rel:.3e}")


def random_state(setup: Setup, seed=0):
    return problems.random_state(setup, seed=seed)


def smooth_state(setup: Setup, seed=0):
    """Smooth periodic state (a few random-phase sinusoids per field) for
    derivative checks: no cell-to-cell noise, so a small perturbation rarely
    crosses a limiter or wave-speed switch."""
    rng = np.random.default_rng(seed)
    u, b, psi = problems._empty(setup)
    x, y, z = (problems._centres(setup, d) for d in range(3))
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    L = [setup.xmax[d] - setup.xmin[d] for d in range(3)]

    def wave(amp):
        k = rng.integers(1, 3, size=3) * [int(setup.n[d] > 1) for d in range(3)]
        ph = rng.uniform(0, 2 * np.pi, size=3)
        return amp * (np.sin(2 * np.pi * k[0] * X / L[0] + ph[0]) * np.cos(2 * np.pi * k[1] * Y / L[1] + ph[1])
                      + np.sin(2 * np.pi * k[2] * Z / L[2] + ph[2]))

    emag = None
    if setup.magnetic:
        for d in range(3):
            b[..., d] = (0.5 if d == 0 else 0.2) + wave(0.15)
        psi[...] = wave(0.02)
        emag = 0.5 * (b ** 2).sum(-1)
    for f, (kind, gam) in enumerate(setup.fluids):
        rho = 1.0 + wave(0.2)
        p = 0.8 + wave(0.15)
        problems._set_fluid(setup, u, f, rho, wave(0.3), wave(0.3), wave(0.3), p,
                            emag if kind == "ion" else None)
    return u, b, psi


def to_soa(setup: Setup, u, b, psi):
    """(u, b, psi) in the guard-cell layout -> one (nplanes, ez, ey, ex) array."""
    planes = [np.moveaxis(u, -1, 0)]
    if setup.magnetic:
        planes += [np.moveaxis(b, -1, 0), psi[None]]
    return np.ascontiguousarray(np.concatenate(planes, 0))


def from_soa(setup: Setup, x):
    nv = setup.nvar
    if setup.magnetic:
        return x[:nv], x[nv:nv + 3], x[nv + 3]
    return x[:nv], None, None
