"""Shared helpers of the test-suite: one state, two engines (oracle and CUDA)."""
import numpy as np

from piernik_b200.config import Setup
from piernik_b200 import problems


def setup_for(phys: str, n=(12, 10, 8), lim="vanleer", limb=None, bnd=None, **kw) -> Setup:
    mag = phys == "mhd"
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
