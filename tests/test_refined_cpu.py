"""Refined (multi-level) domains on the CPU.

The oracle's multi-level driver (oracle/amr.py) is pinned by conservation:
with the fine->coarse flux correction every conserved quantity summed over
leaf cells (times the cell volume) is constant to round-off on a periodic
domain.  The library's planner (pk_levels.cpp, through a host harness) must
produce exactly the couplings the oracle derives independently from cell
positions: the prolonged guard cells with their coarse sources and
parities, the restricted coarse faces with their fine faces in summation
order, and the leaf cells.
"""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from helpers import setup_for
import amr
from piernik_b200 import problems

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "native", "levels_harness.cpp")
PLAN = os.path.join(HERE, "..", "piernik_b200", "csrc", "pk_levels.cpp")
HDR = os.path.join(HERE, "..", "piernik_b200", "csrc", "pk_levels.h")
LIB = os.path.join(HERE, "native", "liblevels_harness.so")
XPLAN = os.path.join(HERE, "..", "piernik_b200", "csrc", "pk_exchange.cpp")

DOM3 = (16, 16, 16)
REG3 = [((8, 8, 8), (24, 24, 24)), ((24, 24, 24), (40, 40, 40))]
DOM2 = (16, 16, 1)
REG2 = [((8, 6, 0), (24, 22, 1)), ((22, 18, 0), (38, 34, 1))]
GO1, GO2 = (1, 0, 0), (2, 2, 1)
RO1, RO2 = (1, 2, 0), (2, 0, 1)


def case(phys, dom=DOM3, regions=REG3, lim="vanleer", seed=3):
    layout = problems.refined_layout(dom, regions, sizes=(8, 16), seed=seed)
    setup = setup_for(phys, n=tuple(8 if d > 1 else 1 for d in dom), lim=lim)
    return problems.refined_blocks(dom, layout, setup, problems.wave_fields(dom, seed=5))


@pytest.fixture(scope="module")
def hlib():
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(f) for f in (SRC, PLAN, HDR, XPLAN)):
        subprocess.check_call(["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-o", LIB, SRC, PLAN, XPLAN])
    L = C.CDLL(LIB)
    L.lv_nruns.restype = C.c_longlong
    L.lv_run.argtypes = [C.c_longlong, C.POINTER(C.c_int)]
    L.lv_fc_slot.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_longlong]
    L.lv_leaf_cells.restype = C.c_longlong
    return L


def build(hlib, blocks, dom):
    nb = len(blocks)
    lev = (C.c_int * nb)(*[b[1] for b in blocks])
    n = (C.c_int * (3 * nb))(*[x for b in blocks for x in b[0].n])
    g = (C.c_int * (3 * nb))(*[x for b in blocks for x in b[0].guards])
    off = (C.c_longlong * (3 * nb))(*[x for b in blocks for x in b[2]])
    dm = (C.c_longlong * 3)(*dom)
    err = C.create_string_buffer(256)
    if hlib.lv_build(nb, lev, n, g, off, dm, err, 256) != 0:
        raise ValueError(err.value.decode())


@pytest.mark.parametrize("phys", ["hd", "mhd"])
@pytest.mark.parametrize("dim", [2, 3])
def test_refined_oracle_conserves(oracle_lib, phys, dim):
    dom, reg = (DOM3, REG3) if dim == 3 else (DOM2, REG2)
    a = amr.AmrOracle(dom, case(phys, dom, reg))
    a.fill_guards()
    t0 = amr.leaf_totals(a)
    scale = amr.leaf_totals(a, absolute=True)
    a.run(2)
    t1 = amr.leaf_totals(a)
    assert a.state.nstep == 2 and a.state.t > 0
    assert np.all(np.abs(t1 - t0) <= 1e-12 * scale), (t1 - t0) / scale


@pytest.mark.parametrize("phys", ["hd", "mhd"])
@pytest.mark.parametrize("dim", [2, 3])
def test_refined_oracle_unsplit_conserves(oracle_lib, phys, dim):
    """The unsplit scheme over the levels (fc_fluxes_unsplit: the coarse
    face flux replaced by the restricted fine ones) conserves the leaf
    totals to round-off, and without the replacement it does not."""
    dom, reg = (DOM3, REG3) if dim == 3 else (DOM2, REG2)
    layout = problems.refined_layout(dom, reg, sizes=(8, 16), seed=3)
    setup = setup_for(phys, n=tuple(8 if d > 1 else 1 for d in dom), solver="unsplit", cfl=0.3, cfl_glm=0.3)
    blocks = problems.refined_blocks(dom, layout, setup, problems.wave_fields(dom, seed=5))
    for teeth in (False, True):
        a = amr.AmrOracle(dom, blocks)
        if teeth:
            a.restr = [[[] for _ in lv] for lv in a.restr]
        a.fill_guards()
        t0 = amr.leaf_totals(a)
        scale = amr.leaf_totals(a, absolute=True)
        a.run(2)
        err = np.max(np.abs(amr.leaf_totals(a) - t0) / scale)
        assert a.state.nstep == 2 and a.state.t > 0
        assert (err > 1e-8) if teeth else (err <= 1e-12), (teeth, err)


def test_refined_oracle_without_correction_does_not_conserve(oracle_lib):
    """The check above has teeth: with the fine fluxes never passed to the
    coarse blocks the leaf totals drift far beyond round-off."""
    a = amr.AmrOracle(DOM3, case("hd"))
    a.restr = [[[] for _ in lv] for lv in a.restr]
    a.fill_guards()
    t0 = amr.leaf_totals(a)
    scale = amr.leaf_totals(a, absolute=True)
    a.run(1)
    assert np.max(np.abs(amr.leaf_totals(a) - t0) / scale) > 1e-8


@pytest.mark.parametrize("dim", [2, 3])
def test_planner_matches_oracle(hlib, oracle_lib, dim):
    dom, reg = (DOM3, REG3) if dim == 3 else (DOM2, REG2)
    blocks = case("mhd", dom, reg)
    build(hlib, blocks, dom)
    a = amr.AmrOracle(dom, blocks)
    # prolonged guard cells: (fine block, x, y, z) -> (coarse block, cx, cy, cz, px, py, pz)
    got = {}
    r = (C.c_int * 12)()
    for k in range(hlib.lv_nruns()):
        hlib.lv_run(k, r)
        fb, cb, fx, fy, fz, ln, cx, cy, cz, px, py, pz = list(r)
        for i in range(ln):
            got[(fb, fx + i, fy, fz)] = (cb, cx + ((px + i) >> 1), cy, cz, (px + i) & 1, py, pz)
    want = {}
    for L, i, dst, j, cs, par in a.prolong:
        z, y, x = dst
        for k in range(len(x)):
            want[(i, int(x[k]), int(y[k]), int(z[k]))] = (j, int(cs[0][k]), int(cs[1][k]), int(cs[2][k]),
                                                          int(par[0][k]), int(par[1][k]), int(par[2][k]))
    assert got == want
    # restricted faces: (coarse block, d, side, pencil position) -> (face, [fine (block, side, position)])
    for d in range(3):
        if dom[d] == 1:
            continue
        slots_in, slots_out = {}, {}
        for b, blk in enumerate(blocks):
            n = blk[0].n
            for kind, tab in ((0, slots_in), (1, slots_out)):
                for side in range(2):
                    if hlib.lv_fc_slot(d, b, kind, side, 0) == -2:
                        continue
                    for i2 in range(n[GO2[d]]):
                        for i1 in range(n[GO1[d]]):
                            s = hlib.lv_fc_slot(d, b, kind, side, i1 + n[GO1[d]] * i2)
                            if s >= 0:
                                pos = [0, 0, 0]
                                pos[GO1[d]], pos[GO2[d]] = i1, i2
                                tab[s] = (b, side, tuple(pos))
        got = {}
        rec = (C.c_int * 5)()
        beg = [hlib.lv_fc_in_level_beg(d, L) for L in range(a.maxl + 1)]
        assert beg == sorted(beg) and beg[-1] == hlib.lv_fc_nin(d)
        for s in range(hlib.lv_fc_nin(d)):
            lc = max(L for L in range(a.maxl) if beg[L] <= s)
            assert beg[lc] <= s < beg[lc + 1] and a.level[slots_in[s][0]] == lc, "in slots grouped by coarse level"
            hlib.lv_fc_in(d, s, rec)
            face, src = rec[0], [x for x in list(rec)[1:] if x >= 0]
            got[slots_in[s]] = (face, [slots_out[x] for x in src])
        want = {}
        for Lc in range(a.maxl + 1):
            for j, side, cpen, order in a.restr[d][Lc]:
                nj = blocks[j][0].n

                def coords(pen, nn):
                    pos = [0, 0, 0]
                    pos[RO1[d]], pos[RO2[d]] = pen % nn[RO1[d]], pen // nn[RO1[d]]
                    return tuple(pos)
                face = int(a._tabs[(j, d)]["in_face"][side][cpen])
                want[(j, side, coords(cpen, nj))] = (face, [(i, s, coords(p, blocks[i][0].n)) for i, s, p in order])
        assert got == want, d
    # leaf cells
    for b in range(len(blocks)):
        n = blocks[b][0].n
        cells = n[0] * n[1] * n[2] if a.leaf[b] is None else int(a.leaf[b].sum())
        assert hlib.lv_leaf_cells(b) == cells


def test_planner_rejects(hlib):
    s = setup_for("hd", n=(8, 8, 8))
    base = [(s.replace(n=(16, 16, 16)), 0, (0, 0, 0))]
    odd = base + [(s.replace(n=(8, 8, 8)), 1, (9, 8, 8))]
    with pytest.raises(ValueError, match="even"):
        build(hlib, odd, (16, 16, 16))
    edge = base + [(s.replace(n=(8, 8, 8)), 1, (0, 8, 8))]       # touches the level boundary: fine,
    build(hlib, edge, (16, 16, 16))                              # level 0 covers the periodic domain
    deep = edge + [(s.replace(n=(8, 8, 8)), 2, (0, 18, 18))]     # level 2 beyond its level 1 block
    with pytest.raises(ValueError, match="nested"):
        build(hlib, deep, (16, 16, 16))
    hole = [(s.replace(n=(16, 16, 8)), 0, (0, 0, 0))]
    with pytest.raises(ValueError, match="cover"):
        build(hlib, hole, (16, 16, 16))


@pytest.mark.parametrize("dim", [2, 3])
def test_refined_oracle_restriction_matches_leaves(oracle_lib, dim):
    """After restriction every covered coarse cell is the mean of its
    children, so the base level alone holds the leaf totals (to round-off),
    after steps that made the levels drift apart."""
    dom, reg = (DOM3, REG3) if dim == 3 else (DOM2, REG2)
    a = amr.AmrOracle(dom, case("mhd", dom, reg))
    a.fill_guards()
    a.run(2)
    leaf = amr.leaf_totals(a)
    scale = amr.leaf_totals(a, absolute=True)

    def base_totals():
        t = None
        for i, ob in enumerate(a.blocks):
            if a.level[i]:
                continue
            s = ob.setup
            g, n = s.guards, s.n
            sl = (slice(g[2], g[2] + n[2]), slice(g[1], g[1] + n[1]), slice(g[0], g[0] + n[0]))
            vol = float(np.prod([s.dl[d] for d in range(3) if a.has[d]]))
            x = np.concatenate([ob.u[sl].reshape(-1, s.nvar).sum(0), ob.b[sl].reshape(-1, 3).sum(0)]) * vol
            t = x if t is None else t + x
        return t
    assert np.max(np.abs(base_totals() - leaf) / scale) > 1e-10      # drifted before
    a.restrict()
    assert np.all(np.abs(base_totals() - leaf) <= 1e-12 * scale)


# level-2 blocks of a refinement update inside the level-1 box of REG3[0]
NEW2 = [((24, 24, 24), (8, 8, 8)), ((32, 24, 24), (8, 8, 8))]


def new_blocks(blocks, placements, dom=DOM3, level=2):
    made = problems.refined_blocks(dom, [(level, off, n) for off, n in placements], blocks[0][0],
                                   problems.wave_fields(dom, seed=5))
    return [(s, L, off) for s, L, off, *_ in made]


def fill_runs(hlib, blocks, dom, target):
    nb = len(blocks)
    lev = (C.c_int * nb)(*[b[1] for b in blocks])
    n = (C.c_int * (3 * nb))(*[x for b in blocks for x in b[0].n])
    g = (C.c_int * (3 * nb))(*[x for b in blocks for x in b[0].guards])
    off = (C.c_longlong * (3 * nb))(*[x for b in blocks for x in b[2]])
    dm = (C.c_longlong * 3)(*dom)
    err = C.create_string_buffer(256)
    hlib.lv_fill.restype = C.c_longlong
    cnt = hlib.lv_fill(nb, lev, n, g, off, dm, target, err, 256)
    if cnt < 0:
        raise ValueError(err.value.decode())
    out = []
    r = (C.c_int * 12)()
    hlib.lv_fill_run.argtypes = [C.c_longlong, C.POINTER(C.c_int)]
    for i in range(cnt):
        hlib.lv_fill_run(i, r)
        out.append(tuple(r))
    return out


def test_planner_fill_runs(hlib, oracle_lib):
    """The rows filling a new block cover its interior once, each cell with
    the parent and parity the oracle's ownership maps give."""
    base = case("hd", DOM3, REG3[:1])
    a = amr.AmrOracle(DOM3, base).relayout(add=new_blocks(base, NEW2))
    blocks = [(ob.setup, a.level[i], a.off[i]) for i, ob in enumerate(a.blocks)]
    for target in (len(blocks) - 2, len(blocks) - 1):
        s = blocks[target][0]
        g, n, off = s.guards, s.n, blocks[target][2]
        seen = {}
        for fb, cb, fx, fy, fz, ln, cx, cy, cz, px, py, pz in fill_runs(hlib, blocks, DOM3, target):
            assert fb == target
            for i in range(ln):
                key = (fx + i, fy, fz)
                assert key not in seen
                seen[key] = (cb, cx + ((px + i) >> 1), cy, cz, (px + i) & 1, py, pz)
        assert len(seen) == n[0] * n[1] * n[2]
        for (x, y, z), got in seen.items():
            F = [x - g[0] + off[0], y - g[1] + off[1], z - g[2] + off[2]]
            P = [f // 2 for f in F]
            j = int(a._owner(1, [np.array(p) for p in P]))
            sj = a.blocks[j].setup
            want = (j,) + tuple(P[d] - a.off[j][d] + sj.guards[d] for d in range(3)) + tuple(f & 1 for f in F)
            assert got == want
    with pytest.raises(ValueError, match="outside"):
        fill_runs(hlib, blocks[:-2] + [(blocks[-1][0], 2, (0, 0, 0))], DOM3, len(blocks) - 2)
    with pytest.raises(ValueError, match="base-level"):
        fill_runs(hlib, blocks, DOM3, 0)


def test_regrid_oracle_restores_by_restriction(oracle_lib):
    """A block filled by the refinement update (u and B injected) restricts
    back to the coarse cells it came from: the eight equal children summed
    one by one round at most in the last bits; cells not covered stay as
    they were."""
    base = case("mhd", DOM3, REG3[:1])
    a = amr.AmrOracle(DOM3, base)
    a.fill_guards()
    a.run(1)
    r = a.relayout(add=new_blocks(base, NEW2))
    r.fill_guards()
    before = [(ob.u.copy(), ob.b.copy()) for ob in r.blocks]
    for k in (len(r.blocks) - 2, len(r.blocks) - 1):
        r.prolong_block(k)
        ob = r.blocks[k]
        g, n = ob.setup.guards, ob.setup.n
        inner = ob.u[g[2]:g[2] + n[2], g[1]:g[1] + n[1], g[0]:g[0] + n[0]]
        assert np.all(np.isfinite(inner)) and np.any(inner != 0.0)
    r.restrict()
    for i, ob in enumerate(r.blocks):
        if r.level[i] == 1:
            for now, was in ((ob.u, before[i][0]), (ob.b, before[i][1])):
                assert np.all(np.abs(now - was) <= 4e-16 * np.abs(was)), i
            changed = np.any(ob.u != before[i][0], axis=-1)
            assert changed.sum() <= 8 * 8 * 8 // 8 * 2, i      # only the cells under the two new blocks


def _cells_of_segs(rows):
    """(block, x, y, z) -> (src block, sx, sy, sz) of copy rows (dst, src, lo, hi, shift)"""
    out = {}
    for dst, src, lx, ly, lz, hx, hy, hz, sx, sy, sz in rows:
        for z in range(lz, hz):
            for y in range(ly, hy):
                for x in range(lx, hx):
                    out[(dst, x, y, z)] = ("copy", src, x + sx, y + sy, z + sz)
    return out


def _cells_of_runs(rows):
    out = {}
    for fb, cb, fx, fy, fz, ln, cx, cy, cz, px, py, pz in rows:
        for i in range(ln):
            out[(fb, fx + i, fy, fz)] = ("prolong", cb, cx + ((px + i) >> 1), cy, cz, (px + i) & 1, py, pz)
    return out


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("r", [1, 2])
def test_partial_refresh_plan(hlib, oracle_lib, dim, r):
    """The guard refresh before a stage along dir writes, with the sources the
    complete refresh uses, every guard cell the stage reads (two layers along
    dir, across the interior) and every coarse guard cell within r of a
    prolonged cell's parent; nothing else is written differently."""
    dom, reg = (DOM3, REG3) if dim == 3 else (DOM2, REG2)
    blocks = case("mhd", dom, reg)
    build(hlib, blocks, dom)
    dm = (C.c_longlong * 3)(*dom)
    ns = hlib.lv_segs(dm)
    assert ns > 0
    row = (C.c_int * 12)()
    hlib.lv_seg.argtypes = [C.c_longlong, C.POINTER(C.c_int)]
    full = {}
    for i in range(ns):
        hlib.lv_seg(i, row)
        full.update(_cells_of_segs([tuple(row[:11])]))
    runs = []
    for i in range(hlib.lv_nruns()):
        hlib.lv_run(i, row)
        runs.append(tuple(row[:12]))
    full.update(_cells_of_runs(runs))
    hlib.lv_partial.restype = C.c_longlong
    hlib.lv_partial_nruns.restype = C.c_longlong
    hlib.lv_partial_seg.argtypes = [C.c_longlong, C.POINTER(C.c_int)]
    hlib.lv_partial_run.argtypes = [C.c_longlong, C.POINTER(C.c_int)]
    has = [d > 1 for d in dom]
    for dr in [d for d in range(3) if has[d]]:
        nps = hlib.lv_partial(dr, r)
        part = {}
        for i in range(nps):
            hlib.lv_partial_seg(i, row)
            part.update(_cells_of_segs([tuple(row[:11])]))
        pruns = []
        for i in range(hlib.lv_partial_nruns()):
            hlib.lv_partial_run(i, row)
            pruns.append(tuple(row[:12]))
        part.update(_cells_of_runs(pruns))
        assert len(part) < len(full)
        for key, src in part.items():                       # the same source as the complete refresh
            assert full[key] == src, key
        for b, (s, L, off, *_) in enumerate(blocks):        # every slab cell
            g, n = s.guards, s.n
            for side in (0, 1):
                lo = [g[d] for d in range(3)]
                hi = [g[d] + n[d] for d in range(3)]
                lo[dr] = g[dr] - 2 if side == 0 else g[dr] + n[dr]
                hi[dr] = lo[dr] + 2
                for z in range(lo[2], hi[2]):
                    for y in range(lo[1], hi[1]):
                        for x in range(lo[0], hi[0]):
                            if (b, x, y, z) in full:
                                assert (b, x, y, z) in part, (dr, b, x, y, z)
        for key, src in part.items():                       # the prolongation stencils' coarse guard cells
            if src[0] != "prolong":
                continue
            _, cb, cx, cy, cz = src[:5]
            sc = blocks[cb][0]
            rr = [r if has[d] else 0 for d in range(3)]
            for z in range(cz - rr[2], cz + rr[2] + 1):
                for y in range(cy - rr[1], cy + rr[1] + 1):
                    for x in range(cx - rr[0], cx + rr[0] + 1):
                        c = (x, y, z)
                        inner = all(sc.guards[d] <= c[d] < sc.guards[d] + sc.n[d] for d in range(3))
                        if not inner and (cb, x, y, z) in full:
                            assert (cb, x, y, z) in part, (dr, key, cb, c)
