"""Refinement criteria and refinement candidates -- TEST INFRASTRUCTURE, NOT
PRODUCT CODE.

A numpy restatement of PIERNIK's unified refinement criteria on a variable
(src/grid/refinement/URC_var.F90) and of the conversion of a block's flag
map into the list of finer blocks to create (refinemap2SFC_list,
src/grid/grid_container_ref.F90:96-142).  Every expression keeps the
reference's operand order (element-wise IEEE operations, no fused
multiply-adds), so the flags are comparable bit for bit.  Parity with the
Fortran is unpinned: the reference holds no known answers for these routines.

Arrays are [z, y, x] with guard cells; ``has`` marks the directions with
extent.  Only tests import this module.
"""
from __future__ import annotations

import numpy as np

THRESHOLD, GRAD, RELGRAD, LOECHNER = 0, 1, 2, 3


def _shifted(p, lo, hi, o):
    """p over the box [lo, hi) (x, y, z) moved by the offset o (x, y, z)."""
    return p[lo[2] + o[2]:hi[2] + o[2], lo[1] + o[1]:hi[1] + o[1], lo[0] + o[0]:hi[0] + o[0]]


def loechner(p, lo, hi, idl, has, aux):
    """refine_on_second_derivative (URC_var.F90:348-437) over the box."""
    e = [tuple(int(has[d] and d == k) for k in range(3)) for d in range(3)]

    def add(a, b):
        return tuple(a[k] + b[k] for k in range(3))

    def neg(a):
        return tuple(-x for x in a)

    def P(o):
        return _shifted(p, lo, hi, o)

    def du(d, o):            # dux / duy / duz at offset o (:447-475)
        return (P(add(o, e[d])) - P(add(o, neg(e[d])))) * idl[d]

    def dau(d, o):           # daux / dauy / dauz at offset o (:461-505)
        return (np.abs(P(add(o, e[d]))) + np.abs(P(add(o, neg(e[d]))))) * idl[d]

    def den(s, t):
        return ((np.abs(du(s, e[t])) + np.abs(du(s, neg(e[t])))) + aux * (dau(s, e[t]) + dau(s, neg(e[t])))) * idl[t]

    def num(s, t):
        return (du(s, e[t]) - du(s, neg(e[t]))) * idl[t]

    shape = P((0, 0, 0)).shape
    sn = np.zeros(shape)
    sd = np.zeros(shape)
    for s in range(3):
        if not has[s]:
            continue
        t = num(s, s)
        a = den(s, s)
        sn = sn + t * t
        sd = sd + a * a
        for c in range(s + 1, 3):          # the mixed terms of s with the later directions
            if not has[c]:
                continue
            t = num(s, c)
            sn = sn + 2.0 * (t * t)
            a = den(s, c)
            b = den(c, s)
            sd = (sd + a * a) + b * b
    with np.errstate(divide="ignore", invalid="ignore"):
        r = np.where(sd > 0.0, sn / np.where(sd > 0.0, sd, 1.0), np.where(sn > 0.0, 1.0, 0.0))
    return r


def _rel1(a, b):
    """rel_grad_1pair (URC_var.F90:674-688)"""
    ok = (np.abs(a) != 0.0) & (np.abs(b) != 0.0)
    with np.errstate(divide="ignore", invalid="ignore"):
        return np.where(ok, np.abs(a - b) / np.where(ok, np.abs(a) + np.abs(b), 1.0), 0.0)


def _sumsq01(a, b):
    """sumsq01 (URC_var.F90:690-706)"""
    return (a * a) * (1.0 - b * b) + b * b


def mark_block(p, n, g, dl, has, level, crits):
    """The flag map (uint8, like p) of one block: crits = [(method, p_field
    array, thr, aux)] with each field array shaped like p."""
    ext = p.shape
    m = np.zeros(ext, dtype=np.uint8)
    idl = [1.0 / dl[d] for d in range(3)]
    lo_i = [g[d] for d in range(3)]
    hi_i = [g[d] + n[d] for d in range(3)]
    for method, f, thr, aux in crits:
        if method == LOECHNER:
            lo = [g[d] - (2 if has[d] else 0) for d in range(3)]
            hi = [g[d] + n[d] + (2 if has[d] else 0) for d in range(3)]
            r = loechner(f, lo, hi, idl, has, aux)
            hit = r >= thr
        else:
            lo, hi = lo_i, hi_i
            P = lambda o: _shifted(f, lo, hi, o)
            e = [tuple(int(has[d] and d == k) for k in range(3)) for d in range(3)]
            if method == THRESHOLD:
                if aux > 0.0 and float(level) >= aux:
                    continue
                hit = P((0, 0, 0)) >= thr
            elif method == GRAD:       # grad2 (:567-580)
                a = P(e[0]) - P(tuple(-x for x in e[0]))
                b = P(e[1]) - P(tuple(-x for x in e[1]))
                c = P(e[2]) - P(tuple(-x for x in e[2]))
                hit = (a * a + b * b) + c * c >= thr * thr
            elif method == RELGRAD:    # rel_grad2 (:645-668)
                c0 = P((0, 0, 0))
                r = np.zeros(c0.shape)
                for d in range(3):
                    if not has[d]:
                        continue
                    pair = _sumsq01(_rel1(c0, P(e[d])), _rel1(c0, P(tuple(-x for x in e[d]))))
                    r = pair if d == 0 else _sumsq01(r, pair)
                hit = r >= thr * thr
            else:
                raise ValueError(method)
        sl = m[lo[2]:hi[2], lo[1]:hi[1], lo[0]:hi[0]]
        sl |= hit.astype(np.uint8)
    return m


def field_of(ob, f):
    """Plane f of an oracle block: u components, then B, then psi."""
    nv = ob.u.shape[-1]
    if f < nv:
        return np.ascontiguousarray(ob.u[..., f])
    if f < nv + 3:
        return np.ascontiguousarray(ob.b[..., f - nv])
    return ob.psi


def mark_amr(a, criteria):
    """pk_mark_refinement over an AmrOracle (guard cells current): maps and
    the per-block 'a leaf interior cell is flagged' answers."""
    maps, flagged = [], []
    for i, ob in enumerate(a.blocks):
        s = ob.setup
        leaf = a.leaf[i]
        if leaf is not None and not leaf.any():
            maps.append(np.zeros(ob.psi.shape if ob.psi is not None else ob.u.shape[:3], dtype=np.uint8))
            flagged.append(0)
            continue
        crits = [(m, field_of(ob, f), thr, aux) for m, f, thr, aux in criteria]
        mp = mark_block(crits[0][1] if crits else ob.u[..., 0], s.n, s.guards, s.dl, a.has, a.level[i], crits)
        g, n = s.guards, s.n
        inner = mp[g[2]:g[2] + n[2], g[1]:g[1] + n[1], g[0]:g[0] + n[0]].astype(bool)
        if leaf is not None:
            inner &= leaf.astype(bool)
        maps.append(mp)
        flagged.append(int(inner.any()))
    return maps, flagged


def candidates(mp, leaf, n, g, off, bsize, has):
    """refinemap2SFC_list (grid_container_ref.F90:96-142) of one block."""
    m = mp.copy()
    inner = m[g[2]:g[2] + n[2], g[1]:g[1] + n[1], g[0]:g[0] + n[0]]
    if leaf is not None:
        inner &= leaf
    if not m.any():
        return []
    if any(has[d] and bsize[d] <= 0 for d in range(3)):
        return []
    bs = [bsize[d] if has[d] else 1 << 40 for d in range(3)]
    is_ = [off[d] for d in range(3)]
    ie = [off[d] + n[d] - 1 for d in range(3)]
    out = []

    def rng(d):
        for i in range((is_[d] * 2) // bs[d], (ie[d] * 2 + 1) // bs[d] + 1):
            yield i, max(is_[d], (i * bs[d]) // 2), min(ie[d], ((i + 1) * bs[d] - 1) // 2)

    for i, ifs, ife in rng(0):
        for j, jfs, jfe in rng(1):
            for k, kfs, kfe in rng(2):
                box = inner[kfs - off[2]:kfe - off[2] + 1, jfs - off[1]:jfe - off[1] + 1, ifs - off[0]:ife - off[0] + 1]
                if box.any():
                    out.append((i * bs[0] if has[0] else 0, j * bs[1] if has[1] else 0, k * bs[2] if has[2] else 0))
    return out
