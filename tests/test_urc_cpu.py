"""The refinement-criteria oracle (oracle/urc.py) on the CPU: known answers
of each criterion on simple fields, and refinemap2SFC_list's candidates
against a direct count over the finer level's blocks."""
import numpy as np
import pytest

import urc

HAS3 = (True, True, True)


def field(fn, n=8, g=4):
    z, y, x = np.meshgrid(*[np.arange(n + 2 * g, dtype=float) - g] * 3, indexing="ij")
    return fn(x, y, z)


def test_loechner_zero_on_linear_and_positive_on_curved():
    n, g = 8, 4
    lin = field(lambda x, y, z: 3.0 * x - 2.0 * y + z + 7.0)
    r = urc.loechner(lin, [g - 2] * 3, [g + n + 2] * 3, [1.0] * 3, HAS3, 0.01)
    assert r.shape == (n + 4,) * 3 and np.all(r == 0.0)
    quad = field(lambda x, y, z: (x - 3.5) ** 2 + 0.5 * y * z + 10.0)
    r = urc.loechner(quad, [g - 2] * 3, [g + n + 2] * 3, [1.0] * 3, HAS3, 0.01)
    assert np.all((r > 0.0) & (r <= 1.0))


def test_loechner_constant_zero_field():
    z = field(lambda x, y, z: 0.0 * x)
    r = urc.loechner(z, [2] * 3, [14] * 3, [1.0] * 3, HAS3, 0.01)
    assert np.all(r == 0.0)                       # sd == 0 and sn == 0: "most likely constant field"


def test_relgrad_and_grad_and_threshold():
    n, g = 8, 4
    c = field(lambda x, y, z: 2.0 + 0.0 * x)
    crits = [(urc.RELGRAD, c, 1e-6, 0.0), (urc.GRAD, c, 1e-6, 0.0)]
    m = urc.mark_block(c, (n,) * 3, (g,) * 3, (1.0,) * 3, HAS3, 0, crits)
    assert not m.any()                            # a constant field flags nothing
    step = field(lambda x, y, z: np.where(x < 4, 1.0, 3.0))
    m = urc.mark_block(step, (n,) * 3, (g,) * 3, (1.0,) * 3, HAS3, 0, [(urc.GRAD, step, 1.5, 0.0)])
    inner = m[g:g + n, g:g + n, g:g + n]
    assert inner[..., 3].all() and inner[..., 4].all() and inner.sum() == 2 * n * n   # (3 - 1)^2 = 4 >= 1.5^2
    # |1 - 3| / 4 = 0.5 along x; the reference's nesting squares the running
    # value at each further direction: 0.5 (+) 0 -> 0.25, then 0.25^2, then
    # 0.0625^2 = 0.00390625 against thr^2
    m = urc.mark_block(step, (n,) * 3, (g,) * 3, (1.0,) * 3, HAS3, 0, [(urc.RELGRAD, step, 0.06, 0.0)])
    assert m[g:g + n, g:g + n, g:g + n].sum() == 2 * n * n
    m = urc.mark_block(step, (n,) * 3, (g,) * 3, (1.0,) * 3, HAS3, 0, [(urc.RELGRAD, step, 0.07, 0.0)])
    assert not m.any()
    m = urc.mark_block(step, (n,) * 3, (g,) * 3, (1.0,) * 3, HAS3, 0, [(urc.THRESHOLD, step, 2.0, 0.0)])
    assert m[g:g + n, g:g + n, g:g + n].sum() == 4 * n * n and m.sum() == 4 * n * n   # interior only
    m = urc.mark_block(step, (n,) * 3, (g,) * 3, (1.0,) * 3, HAS3, 2, [(urc.THRESHOLD, step, 2.0, 2.0)])
    assert not m.any()                            # level 2 >= aux: skipped


@pytest.mark.parametrize("seed", range(4))
def test_candidates_against_direct_count(seed):
    rng = np.random.default_rng(seed)
    n, g = (12, 8, 16), (4, 4, 4)
    off = (6, 10, 4)
    bsize = (8, 4, 8)
    mp = np.zeros((n[2] + 8, n[1] + 8, n[0] + 8), dtype=np.uint8)
    mp[rng.random(mp.shape) < 0.01] = 1
    leaf = (rng.random((n[2], n[1], n[0])) < 0.8).astype(np.uint8)
    got = urc.candidates(mp, leaf, n, g, off, bsize, HAS3)
    inner = mp[4:4 + n[2], 4:4 + n[1], 4:4 + n[0]] & leaf
    want = []
    for fx in range(0, 2 * (off[0] + n[0]) + bsize[0], bsize[0]):
        for fy in range(0, 2 * (off[1] + n[1]) + bsize[1], bsize[1]):
            for fz in range(0, 2 * (off[2] + n[2]) + bsize[2], bsize[2]):
                lo = [max(o, f // 2) for o, f in zip(off, (fx, fy, fz))]
                hi = [min(o + m, (f + b + 1) // 2) for o, m, f, b in zip(off, n, (fx, fy, fz), bsize)]
                if any(l >= h for l, h in zip(lo, hi)):
                    continue
                if inner[lo[2] - off[2]:hi[2] - off[2], lo[1] - off[1]:hi[1] - off[1], lo[0] - off[0]:hi[0] - off[0]].any():
                    want.append((fx, fy, fz))
    assert got == want and len(got) > 0
    assert urc.candidates(mp, leaf, n, g, off, (0, 4, 8), HAS3) == []
