"""Refined (multi-level) restatement of the sweep path -- TEST INFRASTRUCTURE,
NOT PRODUCT CODE.

Drives the oracle's per-block stage (o_solve_cg, with its ext_fluxes hooks)
over blocks on several levels of a periodic domain the way the reference's
sweep does (sweeps.F90:114-279):

* every RK stage solves the finest level first; each fine block records the
  fluxes through its boundary faces that border the coarser level (lo / ro,
  grid_container_fcflx.F90:206-259), which are summed over the 2 x 2 fine
  faces in ORTHO1-outer / ORTHO2-inner order from 0 and scaled by
  1/2**(eff_dim-1) (fc_fluxes.F90:196-231), and replace the coarse block's
  flux through the same face (li / ri, grid_container_fcflx.F90:148-202;
  solve_cg_riemann.F90:353-362);
* after each stage every guard cell whose position lies in an interior of its
  own level is copied from there, and every other guard cell of a refined
  block is prolonged from the next coarser level, coarsest level first
  (cg_leaves.F90:299-347): u by injection, B and psi by the O_I2 stencil
  applied along x, then y, then z (grid_container_prolong.F90:180-453);
* time_step reduces over leaf cells only (timestep.F90:463) and the GLM
  scalars are the min / max over all blocks (hdc.F90:112-138, 310-332).

The couplings are derived here from dense per-level ownership maps of cell
positions, independently of the library's planner.  Only tests import this.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

import oracle as O

# the directional prolongation stencils (grid_container_prolong.F90:223-287):
# order -> ([P_3, P_2, P_1, P0, P1, P2, P3], stencil range)
PROLONG = {
    -6: ([-231 / 65536, 2002 / 65536, -9009 / 65536, 60060 / 65536, 15015 / 65536, -2574 / 65536, 273 / 65536], 3),
    -5: ([0.0, 77 / 8192, -693 / 8192, 6930 / 8192, 2310 / 8192, -495 / 8192, 63 / 8192], 3),
    -4: ([0.0, 35 / 2048, -252 / 2048, 1890 / 2048, 420 / 2048, -45 / 2048, 0.0], 2),
    -3: ([0.0, 0.0, -7 / 128, 105 / 128, 35 / 128, -5 / 128, 0.0], 2),
    -2: ([0.0, 0.0, -3 / 32, 30 / 32, 5 / 32, 0.0, 0.0], 1),
    1: ([0.0, 0.0, 0.0, 3 / 4, 1 / 4, 0.0, 0.0], 1),
    0: ([0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0], 0),
    2: ([0.0, 0.0, -1 / 8, 1.0, 1 / 8, 0.0, 0.0], 1),
    3: ([0.0, 0.0, -5 / 64, 55 / 64, 17 / 64, -3 / 64, 0.0], 2),
    4: ([0.0, 3 / 128, -11 / 64, 1.0, 11 / 64, -3 / 128, 0.0], 2),
    5: ([0.0, 7 / 512, -63 / 512, 462 / 512, 138 / 512, -37 / 512, 5 / 512], 3),
    6: ([-5 / 1024, 44 / 1024, -201 / 1024, 1.0, 201 / 1024, -44 / 1024, 5 / 1024], 3),
}

RO1 = (1, 2, 0)     # pdims ORTHO1 of x, y, z (constants.F90:127-128)
RO2 = (2, 0, 1)


def _floor2(x):
    return np.floor_divide(x, 2)


class AmrOracle:
    """blocks: list of (setup, level, off, u, b, psi); setup of each block
    carries its n and dl (base cell size / 2**level); dom: base-level cells
    (1 where the domain has no extent); every direction with extent is
    periodic."""

    def __init__(self, dom, blocks):
        self.dom = tuple(int(x) for x in dom)
        self.has = tuple(d > 1 for d in self.dom)
        self.eff_dim = sum(self.has)
        self.blocks = []
        self.level = []
        self.off = []
        for setup, lev, off, u, b, psi in blocks:
            self.blocks.append(O.OracleBlock(setup, u, b, psi))
            self.level.append(int(lev))
            self.off.append(tuple(int(x) for x in off))
        self.maxl = max(self.level)
        self.setup0 = blocks[0][0]
        self.mag = self.setup0.magnetic
        self.nv = self.setup0.nvar
        self.fw = self.nv + (4 if self.mag else 0)
        self._owners()
        self._plan_guards()
        self._plan_fluxes()
        self._plan_leaves()
        self.state = O.OState()
        self.state.dt_old = -1.0
        self.state.dt_cur_shrink = 1.0
        self.state.cfl_c = 1.0

    # ---- layout ---------------------------------------------------------
    def grid(self, L):
        return tuple((self.dom[d] << L) if self.has[d] else 1 for d in range(3))

    def _owners(self):
        self.own = []
        for L in range(self.maxl + 1):
            D = self.grid(L)
            m = -np.ones(D[::-1], dtype=np.int64)             # [z, y, x]
            for i, lev in enumerate(self.level):
                if lev != L:
                    continue
                n, o = self.blocks[i].setup.n, self.off[i]
                sl = tuple(slice(o[d], o[d] + n[d]) for d in (2, 1, 0))
                assert (m[sl] < 0).all(), "blocks of one level overlap"
                m[sl] = i
            if L == 0:
                assert (m >= 0).all(), "level 0 must cover the domain"
            self.own.append(m)

    def _wrap(self, L, p):
        D = self.grid(L)
        return tuple(np.mod(p[d], D[d]) for d in range(3))

    def _owner(self, L, p):
        w = self._wrap(L, p)
        return self.own[L][w[2], w[1], w[0]]

    def _guards(self, i):
        """Storage coordinates (x, y, z arrays) of block i's guard cells."""
        s = self.blocks[i].setup
        g, n = s.guards, s.n
        ext = [n[d] + 2 * g[d] for d in range(3)]
        z, y, x = np.meshgrid(*[np.arange(ext[d]) for d in (2, 1, 0)], indexing="ij")
        inner = np.ones(z.shape, bool)
        for d, a in zip(range(3), (x, y, z)):
            inner &= (a >= g[d]) & (a < g[d] + n[d])
        return x[~inner], y[~inner], z[~inner]

    def _plan_guards(self):
        self.copies = []            # (dst block, dst (z,y,x) idx, src block, src idx)
        self.prolong = []           # (level, dst block, dst idx, src block, src centre (x,y,z), parity (x,y,z))
        for i in range(len(self.blocks)):
            s = self.blocks[i].setup
            g = s.guards
            L = self.level[i]
            x, y, z = self._guards(i)
            F = [x - g[0] + self.off[i][0], y - g[1] + self.off[i][1], z - g[2] + self.off[i][2]]
            for d in range(3):
                if not self.has[d]:
                    F[d] = np.zeros_like(F[d])
            own = self._owner(L, F)
            for j in np.unique(own[own >= 0]):
                sel = own == j
                w = self._wrap(L, [F[d][sel] for d in range(3)])
                sj = self.blocks[j].setup
                src = tuple(w[d] - self.off[j][d] + sj.guards[d] for d in (2, 1, 0))
                self.copies.append((i, (z[sel], y[sel], x[sel]), int(j), src))
            if L == 0:
                assert (own >= 0).all()
                continue
            sel = own < 0
            P = [np.where(self.has[d], _floor2(F[d][sel]), 0) for d in range(3)]
            par = [np.where(self.has[d], F[d][sel] - 2 * _floor2(F[d][sel]), 0) for d in range(3)]
            cown = self._owner(L - 1, P)
            assert (cown >= 0).all(), "a refined block is not nested in the coarser level"
            Pw = self._wrap(L - 1, P)
            for j in np.unique(cown):
                m = cown == j
                sj = self.blocks[j].setup
                cs = tuple(Pw[d][m] - self.off[j][d] + sj.guards[d] for d in range(3))
                self.prolong.append((L, i, (z[sel][m], y[sel][m], x[sel][m]), int(j), cs,
                                     tuple(par[d][m] for d in range(3))))

    def _plan_fluxes(self):
        nbk = len(self.blocks)
        self.eflx = [[None] * 3 for _ in range(nbk)]
        self.keep = []
        self.restr = [[[] for _ in range(self.maxl + 1)] for _ in range(3)]   # [d][coarse level]
        tabs = {}

        def tab(i, d):
            if (i, d) not in tabs:
                s = self.blocks[i].setup
                o1, o2 = RO1[d], RO2[d]
                np_ = s.n[o1] * s.n[o2]
                t = {"in_face": [-np.ones(np_, np.int32) for _ in range(2)],
                     "in_flx": [np.zeros((np_, self.fw)) for _ in range(2)],
                     "out_on": [np.zeros(np_, np.int32) for _ in range(2)],
                     "out_flx": [np.zeros((np_, self.fw)) for _ in range(2)]}
                tabs[(i, d)] = t
            return tabs[(i, d)]

        entries = {}
        for i in range(nbk):
            L = self.level[i]
            if L == 0:
                continue
            s = self.blocks[i].setup
            for d in range(3):
                if not self.has[d]:
                    continue
                o1, o2 = RO1[d], RO2[d]
                for side in range(2):
                    for i2 in range(s.n[o2]):
                        for i1 in range(s.n[o1]):
                            F = [0, 0, 0]
                            F[d] = self.off[i][d] - 1 if side == 0 else self.off[i][d] + s.n[d]
                            F[o1] = self.off[i][o1] + i1 if self.has[o1] else 0
                            F[o2] = self.off[i][o2] + i2 if self.has[o2] else 0
                            if self._owner(L, [np.array(v) for v in F]) >= 0:
                                continue
                            pen = i1 + s.n[o1] * i2
                            tab(i, d)["out_on"][side][pen] = 1
                            P = [F[e] // 2 if self.has[e] else 0 for e in range(3)]
                            j = int(self._owner(L - 1, [np.array(v) for v in P]))
                            assert j >= 0
                            Pw = [int(v) for v in self._wrap(L - 1, [np.array(v) for v in P])]
                            sj = self.blocks[j].setup
                            s_out = Pw[d] - self.off[j][d] + sj.guards[d]
                            cpen = (Pw[o1] - self.off[j][o1]) + sj.n[o1] * (Pw[o2] - self.off[j][o2])
                            face = s_out if side == 0 else s_out - 1
                            ct = tab(j, d)
                            assert ct["in_face"][side][cpen] in (-1, face), "two fine regions on one side of a pencil"
                            ct["in_face"][side][cpen] = face
                            pos = 2 * (F[o1] & 1 if self.has[o1] else 0) + (F[o2] & 1 if self.has[o2] else 0)
                            entries.setdefault((j, d, side, cpen), {})[pos] = (i, side, pen)
        for (j, d, side, cpen), srcs in entries.items():
            assert len(srcs) == 2 ** (self.eff_dim - 1)
            order = [srcs[p] for p in sorted(srcs)]
            self.restr[d][self.level[j]].append((j, side, cpen, order))
        self._tabs = tabs
        for (i, d), t in tabs.items():
            e = O_eflx()
            for k in range(2):
                e.in_face[k] = t["in_face"][k].ctypes.data_as(C.POINTER(C.c_int))
                e.in_flx[k] = t["in_flx"][k].ctypes.data_as(C.POINTER(C.c_double))
                e.out_on[k] = t["out_on"][k].ctypes.data_as(C.POINTER(C.c_int))
                e.out_flx[k] = t["out_flx"][k].ctypes.data_as(C.POINTER(C.c_double))
            self.keep.append(e)
            self.blocks[i].blk.eflx[d] = C.addressof(e)

    def _plan_leaves(self):
        self.leaf = [None] * len(self.blocks)
        for i in range(len(self.blocks)):
            L = self.level[i]
            if L == self.maxl:
                continue
            s = self.blocks[i].setup
            z, y, x = np.meshgrid(*[np.arange(s.n[d]) for d in (2, 1, 0)], indexing="ij")
            F = [x + self.off[i][0], y + self.off[i][1], z + self.off[i][2]]
            child = [2 * F[d] if self.has[d] else F[d] for d in range(3)]
            covered = self._owner(L + 1, child) >= 0
            if covered.any():
                m = np.ascontiguousarray((~covered).astype(np.uint8))
                self.leaf[i] = m
                self.blocks[i].blk.leaf = m.ctypes.data

    # ---- one stage's couplings ---------------------------------------------
    def _restrict(self, d, Lc):
        scale = 1.0 / 2.0 ** (self.eff_dim - 1)
        for j, side, cpen, order in self.restr[d][Lc]:
            acc = np.zeros(self.fw)
            for (i, s, pen) in order:
                acc = acc + self._tabs[(i, d)]["out_flx"][s][pen]
            self._tabs[(j, d)]["in_flx"][side][cpen] = scale * acc

    def _chspeed(self, dt):
        """update_chspeed over the leaves (hdc.F90:90-140): the grid bound's
        minimum over blocks, or with ch_grid = .false. the maximum of the
        blocks' leaf-cell point_chspeed maxima"""
        lib, cfg = O.lib(), self.blocks[0].cfg
        vals = [lib.o_chspeed(C.byref(cfg), C.byref(b.blk), dt) for b in self.blocks]
        return min(vals) if cfg.ch_grid else max(vals)

    def fill_guards(self, half=False):
        """update_boundaries of u, b, psi (of uh, bh, psih when ``half``: the
        unsplit scheme's first-stage arrays)"""
        nu, nb, npsi = ("uh", "bh", "psih") if half else ("u", "b", "psi")
        for i, dst, j, src in self.copies:
            A, B = self.blocks[i], self.blocks[j]
            getattr(A, nu)[dst] = getattr(B, nu)[src]
            if self.mag:
                getattr(A, nb)[dst] = getattr(B, nb)[src]
                getattr(A, npsi)[dst] = getattr(B, npsi)[src]
        s0 = self.setup0
        ofl = s0.ord_fluid_prolong if s0.ord_fluid_prolong in (0, 1) else 0
        ku, kb = PROLONG[ofl], PROLONG[s0.ord_mag_prolong]
        pro3 = self._pro3

        for L in range(1, self.maxl + 1):
            for lev, i, dst, j, cs, par in self.prolong:
                if lev != L:
                    continue
                A, B = self.blocks[i], self.blocks[j]
                Au, Bu = getattr(A, nu), getattr(B, nu)
                if ku[1] == 0:
                    Au[dst] = Bu[cs[2], cs[1], cs[0]]
                else:
                    for v in range(Au.shape[-1]):
                        Au[dst + (v,)] = pro3(ku, Bu[..., v], cs, par)
                if not self.mag:
                    continue
                Ab, Bb = getattr(A, nb), getattr(B, nb)
                fields = [(Ab[..., c], Bb[..., c]) for c in range(3)] + [(getattr(A, npsi), getattr(B, npsi))]
                for fa, fb in fields:
                    fa[dst] = pro3(kb, fb, cs, par)

    @staticmethod
    def _pro1(k, get, par):
        """sum over m = -r..r of P(-m) c(m) (left child) or P(m) c(m), left to right"""
        P, r = k
        if r == 0:
            return get(0)
        acc = None
        for m in range(-r, r + 1):
            t = np.where(par == 0, P[3 - m], P[3 + m]) * get(m)
            acc = t if acc is None else acc + t
        return acc

    def _pro3(self, k, fb, cs, par):
        """directional prolongation x, then y, then z (grid_container_prolong.F90:290-453)"""
        pro1 = self._pro1
        r = k[1]
        ry = r if self.has[1] else 0
        rz = r if self.has[2] else 0
        Y = {}
        for kz in range(-rz, rz + 1):
            X = {}
            for ky in range(-ry, ry + 1):
                row = lambda kx, ky=ky, kz=kz: fb[cs[2] + kz, cs[1] + ky, cs[0] + kx]
                X[ky] = pro1(k, row, par[0]) if self.has[0] else row(0)
            Y[kz] = pro1(k, lambda m: X[m], par[1]) if self.has[1] else X[0]
        return pro1(k, lambda m: Y[m], par[2]) if self.has[2] else Y[0]

    def relayout(self, add=(), remove=()):
        """A new driver over this one's blocks minus ``remove`` (ids), plus
        ``add`` = [(setup, level, off)] appended with zero state, carrying
        every remaining block's whole array and the time state."""
        keep = [i for i in range(len(self.blocks)) if i not in set(remove)]
        blocks = []
        for i in keep:
            ob = self.blocks[i]
            blocks.append((ob.setup, self.level[i], self.off[i], ob.u, ob.b, ob.psi))
        for s, lev, off in add:
            ext = (s.ext[2], s.ext[1], s.ext[0])
            blocks.append((s, lev, off, np.zeros(ext + (s.nvar,)), np.zeros(ext + (3,)) if self.mag else None,
                           np.zeros(ext) if self.mag else None))
        new = AmrOracle(self.dom, blocks)
        C.memmove(C.byref(new.state), C.byref(self.state), C.sizeof(O.OState))
        return new

    # ---- filling a new block (refinement update) ----------------------------
    def prolong_block(self, i):
        """Every interior cell of block i (a refined level's) from the level
        below, as cg_level_connected.F90:870-920 / 1059-1093 fill the blocks a
        refinement update creates: u and B (rank-4 arrays) by injection, psi
        at ord_mag_prolong, read from the coarse blocks' storage (guard cells
        included, which must be current)."""
        L = self.level[i]
        assert L >= 1
        A = self.blocks[i]
        s = A.setup
        g, n = s.guards, s.n
        z, y, x = [a.ravel() for a in np.meshgrid(*[np.arange(g[d], g[d] + n[d]) for d in (2, 1, 0)], indexing="ij")]
        F = [x - g[0] + self.off[i][0], y - g[1] + self.off[i][1], z - g[2] + self.off[i][2]]
        P = [np.where(self.has[d], _floor2(F[d]), 0) for d in range(3)]
        par = [np.where(self.has[d], F[d] - 2 * _floor2(F[d]), 0) for d in range(3)]
        cown = self._owner(L - 1, P)
        assert (cown >= 0).all(), "a refined block is not nested in the coarser level"
        Pw = self._wrap(L - 1, P)
        kb = PROLONG[self.setup0.ord_mag_prolong]
        for j in np.unique(cown):
            m = cown == j
            B = self.blocks[int(j)]
            sj = B.setup
            cs = tuple(Pw[d][m] - self.off[j][d] + sj.guards[d] for d in range(3))
            dst = (z[m], y[m], x[m])
            A.u[dst] = B.u[cs[2], cs[1], cs[0]]
            if self.mag:
                A.b[dst] = B.b[cs[2], cs[1], cs[0]]
                A.psi[dst] = self._pro3(kb, B.psi, cs, tuple(par[d][m] for d in range(3)))

    # ---- restriction (restrict_to_base) ---------------------------------
    def restrict(self):
        """Every coarse cell covered by a finer block takes the mean of its
        children, finest level first (cg_level_connected.F90:1395-1409,
        1480-1721): in 3D the eight children summed x fastest, then scaled
        once; otherwise each child scaled and accumulated from 0 in z, y, x
        order; the coarse cell becomes 0 + that."""
        norm = 1.0 / 2.0 ** self.eff_dim
        full3 = self.eff_dim == 3
        for L in range(self.maxl, 0, -1):
            for fi, lf in enumerate(self.level):
                if lf != L:
                    continue
                F = self.blocks[fi]
                sf = F.setup
                lo = [self.off[fi][d] // 2 if self.has[d] else 0 for d in range(3)]
                hi = [(self.off[fi][d] + sf.n[d]) // 2 if self.has[d] else 1 for d in range(3)]
                for ci, lc in enumerate(self.level):
                    if lc != L - 1:
                        continue
                    Cb = self.blocks[ci]
                    sc = Cb.setup
                    a = [max(lo[d], self.off[ci][d]) for d in range(3)]
                    e = [min(hi[d], self.off[ci][d] + sc.n[d]) for d in range(3)]
                    if any(a[d] >= e[d] for d in range(3)):
                        continue
                    cs = tuple(slice(a[d] - self.off[ci][d] + sc.guards[d], e[d] - self.off[ci][d] + sc.guards[d])
                               for d in (2, 1, 0))
                    f0 = [2 * a[d] - self.off[fi][d] + sf.guards[d] if self.has[d] else 0 for d in range(3)]
                    cnt = [e[d] - a[d] for d in range(3)]

                    def child(arr, dx, dy, dz):
                        return arr[f0[2] + dz:f0[2] + dz + 2 * cnt[2]:2 if self.has[2] else 1,
                                   f0[1] + dy:f0[1] + dy + 2 * cnt[1]:2 if self.has[1] else 1,
                                   f0[0] + dx:f0[0] + dx + 2 * cnt[0]:2 if self.has[0] else 1]

                    pairs = [(Cb.u, F.u)] + ([(Cb.b, F.b), (Cb.psi, F.psi)] if self.mag else [])
                    for cA, fA in pairs:
                        if full3:
                            val = (((((((child(fA, 0, 0, 0) + child(fA, 1, 0, 0)) + child(fA, 0, 1, 0))
                                      + child(fA, 1, 1, 0)) + child(fA, 0, 0, 1)) + child(fA, 1, 0, 1))
                                    + child(fA, 0, 1, 1)) + child(fA, 1, 1, 1)) * norm
                        else:
                            val = np.zeros_like(cA[cs])
                            for dz in range(2 if self.has[2] else 1):
                                for dy in range(2 if self.has[1] else 1):
                                    for dx in range(2 if self.has[0] else 1):
                                        val = val + child(fA, dx, dy, dz) * norm
                        cA[cs] = 0.0 + val

    # ---- the main loop ---------------------------------------------------
    def sweep(self, d, dt, ch):
        lib = O.lib()
        nst = 1 if self.setup0.integration_order == 1 else 2
        for st in range(1, nst + 1):
            istep = 1 if nst == 1 else st
            for L in range(self.maxl, -1, -1):
                for i, ob in enumerate(self.blocks):
                    if self.level[i] != L:
                        continue
                    rc = lib.o_solve_cg(C.byref(ob.cfg), C.byref(ob.blk), d, istep, dt, ch)
                    if rc:
                        raise RuntimeError(f"o_solve_cg failed: {rc}")
                if L > 0:
                    self._restrict(d, L - 1)
            self.fill_guards()

    def unsplit_sweep(self, dt, ch):
        """unsplit_sweep (unsplit_sweeps.F90:104-189) over the levels: each
        stage solves the finest level first -- every block's face fluxes of
        all directions with the ext_fluxes hooks, their application and
        sources -- restricting a level's boundary fluxes into the next coarser
        level before it, then updates the boundaries of the array the stage
        wrote (uh, bh, psih after RK2_1)."""
        lib = O.lib()
        nst = 1 if self.setup0.integration_order == 1 else 2
        for st in range(1, nst + 1):
            for L in range(self.maxl, -1, -1):
                for i, ob in enumerate(self.blocks):
                    if self.level[i] != L:
                        continue
                    rc = lib.o_unsplit_stage(C.byref(ob.cfg), C.byref(ob.blk), st, dt, ch)
                    if rc:
                        raise RuntimeError(f"o_unsplit_stage failed: {rc}")
                if L > 0:
                    for d in range(3):
                        if self.has[d]:
                            self._restrict(d, L - 1)
            self.fill_guards(half=(nst == 2 and st == 1))

    def time_step(self):
        lib = O.lib()
        arr = (C.POINTER(O.OBlock) * len(self.blocks))(*[C.pointer(b.blk) for b in self.blocks])
        rc = lib.o_time_step_multi(C.byref(self.blocks[0].cfg), arr, len(self.blocks), C.byref(self.state))
        if rc:
            raise RuntimeError(f"o_time_step_multi failed: {rc}")

    def _glm_fac(self, dt):
        cfg = self.blocks[0].cfg
        f = 0.0
        for b in self.blocks:
            dl = [b.setup.dl[e] for e in range(3) if b.setup.n[e] > 1]
            if dl:
                f = max(f, (cfg.glm_alpha * self.state.chspeed) / (min(dl) / dt))
        return math.exp(-f)

    def fluid_update_unsplit(self):
        """fluid_update_unsplit (unsplit_fluidupdate.F90:45-126) over all blocks"""
        st = self.state
        dt = st.dt
        cfg = self.blocks[0].cfg
        lib = O.lib()
        fac = 1.0
        if self.mag:
            st.chspeed = self._chspeed(dt)
            fac = self._glm_fac(dt / 2.0)
            for b in self.blocks:
                lib.o_glm_apply(C.byref(cfg), C.byref(b.blk), fac)
        st.t = st.t + dt
        self.unsplit_sweep(dt, st.chspeed)
        if self.mag:
            for b in self.blocks:
                lib.o_glm_apply(C.byref(cfg), C.byref(b.blk), fac)

    def fluid_update(self):
        st = self.state
        dt = st.dt
        cfg = self.blocks[0].cfg
        lib = O.lib()
        if self.setup0.solver == "unsplit":
            return self.fluid_update_unsplit()
        if self.mag:
            st.chspeed = self._chspeed(dt)
            f = 0.0
            for b in self.blocks:
                dl = [b.setup.dl[e] for e in range(3) if b.setup.n[e] > 1]
                if dl:
                    f = max(f, (cfg.glm_alpha * st.chspeed) / (min(dl) / dt))
            fac = math.exp(-f)
        for half in range(2):
            st.t = st.t + dt
            for s in range(3):
                d = s if half == 0 else 2 - s
                if cfg.skip_sweep[d] or not self.has[d]:
                    continue
                self.sweep(d, dt, st.chspeed)
            if self.mag:
                for b in self.blocks:
                    lib.o_glm_apply(C.byref(cfg), C.byref(b.blk), fac)

    def run(self, nsteps):
        for _ in range(nsteps):
            self.time_step()
            self.fluid_update()
            self.state.nstep += 1


class O_eflx(C.Structure):
    _fields_ = [("in_face", C.POINTER(C.c_int) * 2), ("in_flx", C.POINTER(C.c_double) * 2),
                ("out_on", C.POINTER(C.c_int) * 2), ("out_flx", C.POINTER(C.c_double) * 2)]


def leaf_totals(amr, absolute: bool = False):
    """Sum over leaf cells of each conserved quantity (of its magnitude when
    ``absolute``) times the cell volume."""
    tot = None
    for i, ob in enumerate(amr.blocks):
        s = ob.setup
        g, n = s.guards, s.n
        sl = (slice(g[2], g[2] + n[2]), slice(g[1], g[1] + n[1]), slice(g[0], g[0] + n[0]))
        vol = float(np.prod([s.dl[d] for d in range(3) if amr.has[d]]))
        m = np.ones(tuple(n[::-1]), bool) if amr.leaf[i] is None else amr.leaf[i].astype(bool)
        f = np.abs if absolute else (lambda x: x)
        t = f(ob.u[sl][m]).sum(0) * vol
        if amr.mag:
            t = np.concatenate([t, f(ob.b[sl][m]).sum(0) * vol])
        tot = t if tot is None else tot + t
    return tot
