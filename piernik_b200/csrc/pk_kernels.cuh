// pk_kernels.cuh -- sweep kernels over pencil tiles staged in shared memory.
//
// Storage of one block on the device (structure of arrays, guard cells kept):
//   u[v][k][j][i], v over the fluid components in flind order, then Bx, By,
//   Bz, psi; i over ext_x = n_x + 2*g_x, etc.  One plane per component.
//
// A CTA owns a tile of P pencils x T cells along the sweep direction; one
// thread per tile cell holds that cell's conservative state in registers for
// the whole launch.  A stage of the reference's pencil solve
// (solve_cg_riemann.F90:318-376) runs as four shared-memory phases separated
// by __syncthreads:
//   1. utoq          -> Q (primitives)
//   2. limited slope -> ql in registers, qr of the cell's left face -> R
//   3. Riemann flux at the cell's right face (own ql, neighbour's R) -> Q
//   4. u1 = u0 + dtodx*(F(i-1/2) - F(i+1/2)), internal_sources, floors
// Which cells do what is decided per thread from its pencil position:
//   * fused mode (periodic single block): both RK2 stages in one launch over a
//     tile with a 4-cell halo read with periodic wrap, output written to a
//     second buffer.  With nb = 4 this equals the reference's stage 1 ->
//     guardcell exchange -> stage 2 bit for bit: every cell the second stage
//     reads was computed from the same inputs by the same operations.
//   * stage mode (any block with guard cells): one stage over a tile with a
//     2-cell halo, pencil ends (the outermost guard cells) handled with the
//     reference's one-sided rules, written back in place.
#pragma once
#include "pk_fast.cuh"

namespace pk {

struct Geom {
    long long plane;        // elements per component plane
    long long sd, s1, s2;   // element strides along the sweep direction and the two ortho directions
    int ext_d;              // pencil length with guards
    int n_d, g_d;           // interior length / guard offset along the sweep direction
    int n1, g1, n2, g2;     // interior extent / guard offset of the ortho directions
    int perm[3];            // slot b+1+j of a swept cell holds plane b+1+perm[j]
    int seg_len = 0;        // independent instances stacked along z: cells per instance (0: one)
    int seg_along = 0;      // 1: this sweep runs along z (the stacking axis)
};

struct Tile {
    int P, T, L;            // pencils, tile length, output cells per pencil
    int xfast;              // 1: lanes run along the pencil (x sweeps)
    int halo;               // stage mode: tile cells before the first owned cell (0 or 2)
    int wrap = 1;           // fused mode: 1 read the halo as periodic images of the interior,
                            // 0 read it from the block's guard cells (filled by the exchange)
    int circ = 0;           // fused mode, periodic block: the tile is the whole pencil (T = L = n)
                            // and cell t's neighbours are t -/+ 1 mod n -- no halo at all
};

// -------------------------------------------------------------------------
// swept load / store of one cell
// -------------------------------------------------------------------------
template <class PH>
PK_DEV int plane_of(int slot, const int (&perm)[3])
{
    // slot -> component plane; fluids [dn, m_n, m_t1, m_t2, en], then B_n, B_t1, B_t2, psi
#pragma unroll
    for (int f = 0; f < PH::NFL; ++f) {
        const int b = PH::beg(f);
        if (slot == b + 1) return b + 1 + perm[0];
        if (slot == b + 2) return b + 1 + perm[1];
        if (slot == b + 3) return b + 1 + perm[2];
    }
    if (PH::MHD) {
        if (slot == PH::IB) return PH::IB + perm[0];
        if (slot == PH::IB + 1) return PH::IB + perm[1];
        if (slot == PH::IB + 2) return PH::IB + perm[2];
    }
    return slot;
}

template <class PH>
PK_DEV void load_cell(const double* u, long long off, const Geom& g, double (&w)[PH::NV])
{
    const int perm[3] = {g.perm[0], g.perm[1], g.perm[2]};
#pragma unroll
    for (int v = 0; v < PH::NV; ++v) w[v] = u[(long long)plane_of<PH>(v, perm) * g.plane + off];
}

template <class PH>
PK_DEV void store_cell(double* u, long long off, const Geom& g, const double (&w)[PH::NV])
{
    const int perm[3] = {g.perm[0], g.perm[1], g.perm[2]};
#pragma unroll
    for (int v = 0; v < PH::NV; ++v) u[(long long)plane_of<PH>(v, perm) * g.plane + off] = w[v];
}

// roles of one tile cell within one stage
struct Roles {
    bool q;        // has a valid input state -> computes primitives
    bool slope;    // computes its limited slope
    int end;       // 0 interior slope, -1 pencil start rule, +1 pencil end rule
    bool flux;     // computes the flux through its right face
    bool upd;      // Euler-updated from the two face fluxes
    bool keep;     // not updated but kept (pencil end cell): u1 = u, then floors
};

// Shared-memory planes of a tile: Q holds primitives and then face fluxes, L
// the left state of each cell's right face, R the right state of its left face.
struct Smem {
    double* Q;
    double* L;
    double* R;
    int PT;
};

// One stage of solve() on the tile.  Nothing but the cell's own state w crosses
// a barrier in registers: primitives and face states live in shared memory and
// the stage's initial state u0 is re-read (from L2) at the update, so the
// Riemann solver runs with a small live set.
//   w      in: the stage's input state (valid where r.q); out: u1 where r.upd or r.keep
//   u0src  where u0 (uh / the sweep's input) is read for the update
//   wsrc   where an unchanged end cell re-reads its state (r.keep)
//   REC    record which floors clipped in *rec (the adjoint sweep's recomputation)
//   me, mp, mn   this cell's slot in the shared planes and its previous / next
//                neighbour's along the pencil (me -/+ the pencil stride, or the
//                wrapped slot in a circular whole-pencil tile)
//   W3     interpol_str = 'weno3' face states (a compile-time choice, so that the
//          limited-linear kernels carry no WENO3 code)
//   FC     fine/coarse flux hooks (ext_fluxes, solve_cg_riemann.F90:353-362): where
//          fc_in is set, the flux through this cell's right face is replaced by
//          the NV values there (li / ri); where fc_out is set, it is stored there
//          (lo / ro), before the update
//   FAST   tolerance-mode arithmetic (pk_fast.cuh): kernels instantiated with it
//          are compiled in their own translation units with contraction on
//   U0S    u0 comes from shared memory (a staged tile): component plane j of
//          this cell at u0sm[j * u0st] instead of u0src in global memory
template <class PH, bool REC = false, bool W3 = false, bool FC = false, bool FAST = false, bool U0S = false>
PK_DEV void rk_stage(const Smem& sm, int me, int mp, int mn, const Roles& r, double (&w)[PH::NV], const double* u0src,
                     const double* wsrc, long long off, const Geom& g, double dtodx, double ch,
                     const PhysParams& pp, unsigned& status, FloorRec* rec = nullptr,
                     const double* fc_in = nullptr, double* fc_out = nullptr, const double* u0sm = nullptr,
                     int u0st = 0)
{
    constexpr int NV = PH::NV;
    const int PT = sm.PT;
    if (r.q) {
        double q[NV];
        if constexpr (FAST) utoq_fast<PH>(w, q, pp);
        else utoq<PH>(w, q, pp);
#pragma unroll
        for (int v = 0; v < NV; ++v) sm.Q[v * PT + me] = q[v];
    }
    __syncthreads();
    if constexpr (W3) {
        if (r.slope) {
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            const double qc = sm.Q[v * PT + me];
            double l = qc, rr = qc;                           // pencil ends: ql(1) = q(1), qr(n-1) = q(n)
            if (r.end == 0) weno3_faces(sm.Q[v * PT + mp], qc, sm.Q[v * PT + mn], pp.w_epsilon, l, rr);
            sm.L[v * PT + me] = l;
            sm.R[v * PT + me] = rr;
        }
        }
    } else if (r.slope) {
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            const int lim = (PH::MHD && v >= PH::IB) ? pp.limb : pp.lim;
            const double qc = sm.Q[v * PT + me];
            double s;
            if (r.end < 0) s = slope_end(lim, sm.Q[v * PT + mn] - qc);
            else if (r.end > 0) s = slope_end(lim, qc - sm.Q[v * PT + mp]);
            else s = slope_interior(lim, qc - sm.Q[v * PT + mp], sm.Q[v * PT + mn] - qc);
            const double dqh = 0.5 * s;                       // dq_interp = half * f_limiter(q)
            sm.L[v * PT + me] = qc + dqh;                     // left state of the right face
            sm.R[v * PT + me] = qc - dqh;                     // right state of the left face
        }
    }
    __syncthreads();
    if (r.flux) {
        if constexpr (FAST) riemann_tile_fast<PH>(sm.L, sm.R, sm.Q, PT, me, mn - me, ch, rcp_nr(ch), pp);
        else riemann_tile<PH>(sm.L, sm.R, sm.Q, PT, me, mn - me, ch, pp);
    }
    __syncthreads();
    if constexpr (FC) {
        if (r.flux && fc_in) {
#pragma unroll
            for (int v = 0; v < NV; ++v) sm.Q[v * PT + me] = __ldcg(fc_in + v);
        }
        if (r.flux && fc_out) {
#pragma unroll
            for (int v = 0; v < NV; ++v) fc_out[v] = sm.Q[v * PT + me];
        }
        __syncthreads();
    }
    if (r.upd) {
        double u0[NV];
        if constexpr (U0S) {
            const int perm[3] = {g.perm[0], g.perm[1], g.perm[2]};
#pragma unroll
            for (int v = 0; v < NV; ++v) u0[v] = u0sm[plane_of<PH>(v, perm) * u0st];
        } else {
            load_cell<PH>(u0src, off, g, u0);
        }
#pragma unroll
        for (int v = 0; v < NV; ++v) w[v] = u0[v] + dtodx * (sm.Q[v * PT + mp] - sm.Q[v * PT + me]);
    } else if (r.keep) {
        load_cell<PH>(wsrc, off, g, w);
    }
    if (r.upd || r.keep) {
        if constexpr (REC) floors_rec<PH>(w, pp, status, *rec);
        else sources_and_floors<PH>(w, pp, status);
    }
    __syncthreads();
}

PK_DEV void flush_status(unsigned status, unsigned* gstatus)
{
    const unsigned s = __reduce_or_sync(0xffffffffu, status);
    if (s && (threadIdx.x & 31) == 0) atomicOr(gstatus, s);
}

PK_DEV int wrap(int s, int n)
{
    int r = s % n;
    return r < 0 ? r + n : r;
}

// Scalars of one step that change from step to step.  Kernels read them from
// device memory so that a captured CUDA graph of the step stays valid.
struct StepParams {
    double dt;        // time step
    double ch;        // GLM psi speed (update_chspeed)
    double psi_fac;   // glmdamping factor, applied by the last sweep of each triple
};

// floor records of both stages of one cell, as the recording sweep stores
// them: bits 0-2 density floors of stage 1 (one per fluid), 3-5 its
// internal-energy floors, 6-8 and 9-11 the same for stage 2
PK_DEV unsigned short pack_floors(const FloorRec& r1, const FloorRec& r2)
{
    return (unsigned short)(r1.dn | (r1.en << 3) | (r2.dn << 6) | (r2.en << 9));
}

// One tile of the fused two-stage sweep of a periodic block (uin -> uout):
// P pencils starting at ortho-1 index i1_0, output cells [c0, c0+L) along the
// sweep, ortho-2 index i2.  The tile reads a 4-cell halo with periodic wrap
// (or is the whole pencil, Tile::circ).  REC: also store the stage-1 state of
// the owned cells in ustar and their floor records in flags (the backward
// pass's recomputation).
template <class PH, bool REC = false, bool W3 = false, bool FAST = false>
PK_DEV void fused_tile(const Geom& g, const Tile& tl, int i1_0, int c0, int i2, const double* uin, double* uout,
                       const PhysParams& pp, const StepParams* __restrict__ sp, double dl, int apply_fac,
                       double* smem, unsigned& status, double* ustar = nullptr, unsigned short* flags = nullptr)
{
    // the step scalars of this tile's instance (one instance unless stacked along z)
    const StepParams stp = sp[g.seg_len ? ((g.seg_along ? c0 : i2) / g.seg_len) : 0];
    const double dtodx1 = (0.5 * stp.dt) / dl;        // rk_coef(RK2_1) * dt / cg%dl(ddim)
    const double dtodx2 = (1.0 * stp.dt) / dl;        // rk_coef(RK2_2) * dt / cg%dl(ddim)
    const double ch = stp.ch, psi_fac = apply_fac ? stp.psi_fac : 1.0;
    constexpr int NV = PH::NV;
    const int P = tl.P, T = tl.T, PT = P * T;
    const Smem sm{smem, smem + NV * PT, smem + 2 * NV * PT, PT};
    const int tid = threadIdx.x;
    int p, t;
    if (tl.xfast) { t = tid % T; p = tid / T; }
    else { p = tid % P; t = tid / P; }
    const int pstride = tl.xfast ? T : 1, st = tl.xfast ? 1 : P;
    const int me = p * pstride + t * st;
    const int i1 = i1_0 + p;
    const bool active = (tid < PT) && (i1 < g.n1);
    const bool circ = tl.circ;
    const int s = circ ? c0 + t : c0 - 4 + t;                  // position along the pencil (interior coords)
    const long long off = (long long)(g.g_d + (tl.wrap ? wrap(s, g.n_d) : s)) * g.sd + (long long)(g.g1 + i1) * g.s1 +
                          (long long)(g.g2 + i2) * g.s2;
    const int mp = circ ? p * pstride + (t == 0 ? T - 1 : t - 1) * st : me - st;
    const int mn = circ ? p * pstride + (t == T - 1 ? 0 : t + 1) * st : me + st;
    double w[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) w[v] = 0.0;
    if (active) load_cell<PH>(uin, off, g, w);
    Roles r;
    r.end = 0;
    r.keep = false;
    const bool own = active && (circ || (t >= 4 && t < T - 4 && s < c0 + tl.L && s < g.n_d));
    FloorRec rec1{0, 0}, rec2{0, 0};
    // both RK2 stages through one copy of the stage code (the solver inlined
    // twice crowds the instruction cache)
#pragma unroll 1
    for (int stage = 0; stage < 2; ++stage) {
        // stage 1 (RK2_1) on tile cells [0, T) (circular: every cell); stage 2
        // (RK2_2) on tile cells [2, T-2), u0 again the sweep's input
        const int a = 2 * stage;
        r.q = active && (circ || (t >= a && t < T - a));
        r.slope = active && (circ || (t >= a + 1 && t < T - a - 1));
        r.flux = active && (circ || (t >= a + 1 && t < T - a - 2));
        r.upd = active && (circ || (t >= a + 2 && t < T - a - 2));
        FloorRec rec{0, 0};
        rk_stage<PH, REC, W3, false, FAST>(sm, me, mp, mn, r, w, uin, uin, off, g, stage == 0 ? dtodx1 : dtodx2, ch,
                                           pp, status, &rec);
        if (stage == 0) {
            rec1 = rec;
            if (REC && own) store_cell<PH>(ustar, off, g, w);
        } else {
            rec2 = rec;
        }
    }
    if (own) {
        if (PH::MHD) w[PH::IB + 3] = w[PH::IB + 3] * psi_fac;   // glmdamping fused into the last sweep
        store_cell<PH>(uout, off, g, w);
        if (REC) flags[off] = pack_floors(rec1, rec2);
    }
}

// -------------------------------------------------------------------------
// Fused two-stage sweep of one periodic block.
// grid: x = ortho-1 tiles of P pencils, y = chunks of L cells, z = ortho-2.
// -------------------------------------------------------------------------
template <class PH, int MAXT, int MINB, bool W3 = false, bool FAST = false>
__global__ void __launch_bounds__(MAXT, MINB) k_sweep_fused(Geom g, Tile tl, const double* __restrict__ uin,
                                                           double* __restrict__ uout, PhysParams pp, double dl,
                                                           const StepParams* __restrict__ sp, int apply_fac,
                                                           unsigned* __restrict__ gstatus)
{
    extern __shared__ double smem[];
    unsigned status = 0;
    fused_tile<PH, false, W3, FAST>(g, tl, blockIdx.x * tl.P, blockIdx.y * tl.L, blockIdx.z, uin, uout, pp, sp, dl, apply_fac,
                              smem, status);
    flush_status(status, gstatus);
}

// -------------------------------------------------------------------------
// Batched fused sweep over many periodic blocks of different sizes: one
// persistent launch; CTAs take tiles from a work list through an atomic
// counter (reset to zero before each launch).
// -------------------------------------------------------------------------
struct BlockDesc {
    const double* in;       // the sweep's input state (structure of arrays with guards)
    double* out;            // where the swept state goes
    long long plane;
    int ext[3], g[3], n[3];
    double dl[3];
    int wrap;               // Tile::wrap for this block's tiles
    const unsigned char* leaf = nullptr;   // interior leaf mask for the CFL reduction (null: every cell)
    double* uh = nullptr;   // stage path: the state at the start of the stage pair (cg%w(uh))
};

struct WorkItem {
    int block;              // index into the block table
    int i1_0, c0, i2;       // first pencil, first output cell, ortho-2 index
    int P, L;               // tile of this item (T = L + 8, or T = L = n when circ)
    int circ;               // whole periodic pencil without halo (Tile::circ)
};

template <class PH, int MAXT, int MINB, bool W3 = false, bool FAST = false>
__global__ void __launch_bounds__(MAXT, MINB) k_sweep_batched(const BlockDesc* __restrict__ blocks,
                                                             const WorkItem* __restrict__ items, int nitems, int dir,
                                                             PhysParams pp, const StepParams* __restrict__ sp,
                                                             int apply_fac, unsigned* __restrict__ counter,
                                                             unsigned* __restrict__ gstatus)
{
    extern __shared__ double smem[];
    __shared__ int next;
    const int o1 = dir == 0 ? 1 : 0, o2 = dir == 2 ? 1 : 2;
    unsigned status = 0;
    for (;;) {
        if (threadIdx.x == 0) next = (int)atomicAdd(counter, 1u);
        __syncthreads();
        const int it = next;
        __syncthreads();
        if (it >= nitems) break;
        const WorkItem w = items[it];
        const BlockDesc b = blocks[w.block];
        Geom g;
        const long long st3[3] = {1, b.ext[0], (long long)b.ext[0] * b.ext[1]};
        g.plane = b.plane;
        g.sd = st3[dir];
        g.s1 = st3[o1];
        g.s2 = st3[o2];
        g.ext_d = b.ext[dir];
        g.n_d = b.n[dir];
        g.g_d = b.g[dir];
        g.n1 = b.n[o1];
        g.g1 = b.g[o1];
        g.n2 = b.n[o2];
        g.g2 = b.g[o2];
        g.perm[0] = dir;                          // iarr_swp: (x,y,z) (y,x,z) (z,y,x)
        g.perm[1] = dir == 1 ? 0 : 1;
        g.perm[2] = dir == 2 ? 0 : 2;
        Tile tl;
        tl.P = w.P;
        tl.L = w.L;
        tl.T = w.circ ? w.L : w.L + 8;
        tl.xfast = dir == 0;
        tl.halo = 4;
        tl.wrap = b.wrap;
        tl.circ = w.circ;
        fused_tile<PH, false, W3, FAST>(g, tl, w.i1_0, w.c0, w.i2, b.in, b.out, pp, sp, b.dl[dir], apply_fac, smem,
                                        status);
    }
    flush_status(status, gstatus);
}

// The fine/coarse flux couplings of one block along one sweep direction.
// Pencils are numbered i1 + n1 * i2; slots index the per-direction arrays
// shared by all blocks.
struct FcArgs {
    const int* in_slot;      // [2][pencils]: slot of the coarse-side override, -1 none
    const int* in_face;      // per in slot: storage index of the cell whose right face takes it
    const double* in_flux;   // per in slot: NV restricted fine fluxes
    const int* out_slot;     // [2][pencils]: slot of the block's own LO / HI boundary face, -1 none
    double* out_flux;        // per out slot: NV fluxes
};

// -------------------------------------------------------------------------
// One RK stage of solve_cg on a tile of a block with guard cells: P pencils
// from ortho-1 index i1_0 at ortho-2 index i2.  The tile spans
// [c0-halo, c0-halo+T) of the pencil: the whole pencil (halo 0, T = L = ext)
// or a chunk with a 2-cell halo; pencil ends (storage index 0 and ext-1)
// follow the reference's one-sided limiter rules and get floors without an
// update, exactly like cells 1 and n of solve().
// first != 0: u0 = u and the owned cells are copied to uh (pu0 = pu).
// uin and uout may alias only when one chunk covers the whole pencil (every
// load of a pencil then precedes every store of it, within one CTA).
// dtodx = rk_coef * dt / dl and ch come from the step scalars in device
// memory, so that a captured CUDA graph serves every step.
// trim: the caller overwrites every guard cell after the stage (the sweeps'
// boundary update), so only the interior cells are updated and stored: the
// tile is then [g-2, g+n+2) of the pencil (c0 = g-2, T = L = n+4), which holds
// every cell the interior updates read.
// -------------------------------------------------------------------------
// The ext_fluxes of storage cell s of pencil (i1, i2): the restricted fine
// flux replacing the flux through its right face (li / ri) and the slot
// recording the flux through it (lo / ro: the faces just outside the interior)
template <class PH>
PK_DEV void fc_slots(const FcArgs& fc, const Geom& g, int i1, int i2, int s, const double*& fc_in, double*& fc_out)
{
    const long long np = (long long)g.n1 * g.n2;
    const long long pen = i1 + (long long)g.n1 * i2;
#pragma unroll
    for (int side = 0; side < 2; ++side) {
        if (fc.in_slot) {
            const int sl = fc.in_slot[side * np + pen];
            if (sl >= 0 && fc.in_face[sl] == s) fc_in = fc.in_flux + (long long)sl * PH::NV;
        }
        if (fc.out_slot) {
            const int sl = fc.out_slot[side * np + pen];
            if (sl >= 0 && s == (side == 0 ? g.g_d - 1 : g.g_d + g.n_d - 1))
                fc_out = fc.out_flux + (long long)sl * PH::NV;
        }
    }
}

template <class PH, bool W3, bool FC>
PK_DEV void stage_tile(const Geom& g, const Tile& tl, int i1_0, int c0, int i2, const double* uin, double* uout,
                       double* uh, const PhysParams& pp, int first, double dtodx, double ch, const FcArgs& fc,
                       double* smem, unsigned& status, bool trim = false, bool flat = false)
{
    constexpr int NV = PH::NV;
    const int P = tl.P, T = tl.T, PT = P * T;
    const Smem sm{smem, smem + NV * PT, smem + 2 * NV * PT, PT};
    const int tid = threadIdx.x;
    int p, t;
    if (tl.xfast) { t = tid % T; p = tid / T; }
    else { p = tid % P; t = tid / P; }
    const int sp = tl.xfast ? T : 1, st = tl.xfast ? 1 : P;
    const int me = p * sp + t * st;
    // flat: the tile's pencils are i1_0 + p in i1-fastest order over the whole
    // block face, so that a CTA may take pencils of consecutive i2 rows
    int i1 = i1_0 + p;
    bool in_face = i1 < g.n1;
    if (flat) {
        in_face = i1 < g.n1 * g.n2;
        i2 = i1 / g.n1;
        i1 -= i2 * g.n1;
    }
    const int n = g.ext_d;
    const int s = c0 - tl.halo + t;                            // storage index along the pencil
    const bool valid = (tid < PT) && in_face && s >= 0 && s < n;
    const bool own = valid && s >= c0 && s < c0 + tl.L;
    const long long off = (long long)s * g.sd + (long long)(g.g1 + i1) * g.s1 + (long long)(g.g2 + i2) * g.s2;
    double w[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) w[v] = 0.0;
    if (valid) load_cell<PH>(uin, off, g, w);
    const bool inner = s >= g.g_d && s < g.g_d + g.n_d;
    if (first && own && (!trim || inner)) store_cell<PH>(uh, off, g, w);   // pu0 = pu (solve_cg_riemann.F90:176)
    Roles r;
    r.q = valid;
    r.end = (s == 0) ? -1 : ((s == n - 1) ? 1 : 0);
    r.slope = valid && (r.end != 0 || (t >= 1 && t <= T - 2));
    // the flux through the right face needs this cell's slope and the next cell's
    const bool next_slope = (s + 1 < n) && (t + 1 <= T - 1) && ((s + 1 == n - 1) || (t + 1 <= T - 2));
    r.flux = r.slope && next_slope;
    // the update needs the left-face flux computed by tile cell t-1
    const bool prev_flux = (t >= 1) && (s >= 1) && ((s - 1 == 0) || (t - 1 >= 1));
    r.upd = valid && s >= 1 && s <= n - 2 && prev_flux && r.flux;
    r.keep = !r.upd && valid && (s == 0 || s == n - 1);        // u1 = u at the pencil ends, then floors
    const double* fc_in = nullptr;
    double* fc_out = nullptr;
    if constexpr (FC)
        if (valid) fc_slots<PH>(fc, g, i1, i2, s, fc_in, fc_out);
    rk_stage<PH, false, W3, FC>(sm, me, me - st, me + st, r, w, first ? uin : uh, uin, off, g, dtodx, ch, pp, status,
                                nullptr, fc_in, fc_out);
    if (own && (!trim || inner)) store_cell<PH>(uout, off, g, w);
}

// One stage of one block.  grid: x = ortho-1 tiles, y = chunks of L cells of
// the full pencil, z = ortho-2.
template <class PH, int MAXT, bool W3 = false, bool FC = false>
__global__ void __launch_bounds__(MAXT) k_stage(Geom g, Tile tl, const double* uin, double* uout, double* uh,
                                               PhysParams pp, int first, double rk, double dl,
                                               const StepParams* __restrict__ spar, unsigned* __restrict__ gstatus,
                                               FcArgs fc = FcArgs{})
{
    extern __shared__ double smem[];
    unsigned status = 0;
    const double dtodx = (rk * spar->dt) / dl;                 // rk_coef(istep) * dt / cg%dl(ddim)
    stage_tile<PH, W3, FC>(g, tl, blockIdx.x * tl.P, blockIdx.y * tl.L, blockIdx.z, uin, uout, uh, pp, first, dtodx,
                           spar->ch, fc, smem, status);
    flush_status(status, gstatus);
}

// One stage of many blocks in one launch: one CTA per work item of P
// pencils (in place, the trimmed tile: every guard cell is refreshed after
// the stage).  blocks[b].in is the state, blocks[b].uh its stage-1 copy; fcs
// (or null) the blocks' flux couplings along dir.
struct StageItem {
    int block, i1_0, i2, P;     // i1_0: first pencil in i1-fastest order over the face (i2 unused)
};

template <class PH, int MAXT, int MINB, bool W3 = false, bool FC = false>
__global__ void __launch_bounds__(MAXT, MINB) k_stage_batched(const BlockDesc* __restrict__ blocks,
                                                       const StageItem* __restrict__ items, int dir, PhysParams pp,
                                                       int first, double rk, const StepParams* __restrict__ spar,
                                                       const FcArgs* __restrict__ fcs, unsigned* __restrict__ gstatus)
{
    extern __shared__ double smem[];
    unsigned status = 0;
    const StageItem w = items[blockIdx.x];
    const BlockDesc b = blocks[w.block];
    const int o1 = dir == 0 ? 1 : 0, o2 = dir == 2 ? 1 : 2;
    Geom g;
    const long long st3[3] = {1, b.ext[0], (long long)b.ext[0] * b.ext[1]};
    g.plane = b.plane;
    g.sd = st3[dir];
    g.s1 = st3[o1];
    g.s2 = st3[o2];
    g.ext_d = b.ext[dir];
    g.n_d = b.n[dir];
    g.g_d = b.g[dir];
    g.n1 = b.n[o1];
    g.g1 = b.g[o1];
    g.n2 = b.n[o2];
    g.g2 = b.g[o2];
    g.perm[0] = dir;                              // iarr_swp: (x,y,z) (y,x,z) (z,y,x)
    g.perm[1] = dir == 1 ? 0 : 1;
    g.perm[2] = dir == 2 ? 0 : 2;
    Tile tl;
    tl.P = w.P;
    tl.T = b.n[dir] + 4;                          // [g-2, g+n+2): the interior updates' stencil
    tl.L = tl.T;
    tl.halo = 0;
    tl.xfast = dir == 0;
    const double dtodx = (rk * spar->dt) / b.dl[dir];
    const FcArgs fc = fcs ? fcs[w.block] : FcArgs{};
    double* u = const_cast<double*>(b.in);
    stage_tile<PH, W3, FC>(g, tl, w.i1_0, b.g[dir] - 2, w.i2, u, u, b.uh, pp, first, dtodx, spar->ch, fc, smem, status,
                           true, true);
    flush_status(status, gstatus);
}

// -------------------------------------------------------------------------
// One RK stage of every block of a refined domain along dir in ONE persistent
// launch (sweeps.F90:218-262: the finer level's boundary fluxes replace the
// coarser level's; the per-level launches do level by level with a
// restriction launch between).  CTAs (occupancy x SMs of them) take work
// items in list order from counters[0]: stage items (P pencils of one block,
// as k_stage_batched) and restriction chunks (in slots [beg, end) of one
// coarse level, as k_restrict_flux).  An item that needs earlier work waits
// until a completion counter reaches its count: a restriction chunk of
// coarse level L-1 for every stage item of level L, a stage item of a block
// with replaced fluxes for every restriction chunk of its level.  The host
// lists every item after all items it waits for, so the earliest unfinished
// item never waits and the launch cannot deadlock while its CTAs are
// resident; the wait is bounded all the same (PK_ST_TIMEOUT after about 4 s,
// the item skipped).  Producers fence their global writes before counting;
// consumers read the replaced and the fine fluxes with L1-bypassing loads.
// Counters: [0] next item, [1 + L] stage items of level L done, [1 + nlev +
// L] restriction chunks for coarse level L done (zeroed before each launch).
// -------------------------------------------------------------------------
struct RefItem {
    int kind;                 // 0 stage item, 1 restriction chunk
    int block, i1_0, P;       // stage item
    int level;                // stage: the block's level; restriction: the coarse level of its slots
    int beg, end;             // restriction: in slots [beg, end)
    int wait;                 // counter to wait on, -1 none
    int wait_count;           // ... until it reaches this
    int fence;                // 1: other items read what it writes (boundary or restricted fluxes)
};

struct RefArgs {
    const int* src;           // 4 fine out slots per in slot (k_restrict_flux's table), -1 none
    const double* out_flux;   // fine boundary fluxes, NV per out slot
    double* in_flux;          // restricted fluxes, NV per in slot
    double scale;             // 1 / 2^(dim-1)
    int nlev;                 // levels
};

template <class PH, int MAXT, int MINB, bool W3 = false>
__global__ void __launch_bounds__(MAXT, MINB) k_stage_refined(const BlockDesc* __restrict__ blocks,
                                                       const RefItem* __restrict__ items, int nitems, int dir,
                                                       PhysParams pp, int first, double rk,
                                                       const StepParams* __restrict__ spar,
                                                       const FcArgs* __restrict__ fcs, RefArgs ra,
                                                       unsigned* __restrict__ counters, unsigned* __restrict__ gstatus)
{
    extern __shared__ double smem[];
    __shared__ int s_item, s_ok;
    constexpr int NV = PH::NV;
    unsigned status = 0;
    const int o1 = dir == 0 ? 1 : 0, o2 = dir == 2 ? 1 : 2;
    // thread 0 claims the next item while the current one runs (an item only
    // waits for items listed before it, so holding a claim cannot block them)
    int claim = threadIdx.x == 0 ? (int)atomicAdd(counters, 1u) : 0;
    for (;;) {
        if (threadIdx.x == 0) {
            const int idx = claim;
            if (idx < nitems) claim = (int)atomicAdd(counters, 1u);
            int ok = 1;
            if (idx < nitems) {
                const int wt = items[idx].wait, wc = items[idx].wait_count;
                if (wt >= 0) {
                    const volatile unsigned* c = counters + wt;
                    for (long long spin = 0; *c < (unsigned)wc; ++spin) {
                        if (spin > (1LL << 26)) {
                            ok = 0;
                            break;
                        }
                        __nanosleep(64);
                    }
                    __threadfence();
                }
            }
            s_item = idx;
            s_ok = ok;
        }
        __syncthreads();
        const int idx = s_item;
        if (idx >= nitems) break;
        if (!s_ok) {
            status |= 4u;                                  // PK_ST_TIMEOUT
            break;
        }
        const RefItem it = items[idx];
        if (it.kind == 0) {
            const BlockDesc b = blocks[it.block];
            Geom g;
            const long long st3[3] = {1, b.ext[0], (long long)b.ext[0] * b.ext[1]};
            g.plane = b.plane;
            g.sd = st3[dir];
            g.s1 = st3[o1];
            g.s2 = st3[o2];
            g.ext_d = b.ext[dir];
            g.n_d = b.n[dir];
            g.g_d = b.g[dir];
            g.n1 = b.n[o1];
            g.g1 = b.g[o1];
            g.n2 = b.n[o2];
            g.g2 = b.g[o2];
            g.perm[0] = dir;                               // iarr_swp: (x,y,z) (y,x,z) (z,y,x)
            g.perm[1] = dir == 1 ? 0 : 1;
            g.perm[2] = dir == 2 ? 0 : 2;
            Tile tl;
            tl.P = it.P;
            tl.T = b.n[dir] + 4;                           // [g-2, g+n+2): the interior updates' stencil
            tl.L = tl.T;
            tl.halo = 0;
            tl.xfast = dir == 0;
            const double dtodx = (rk * spar->dt) / b.dl[dir];
            const FcArgs fc = fcs ? fcs[it.block] : FcArgs{};
            double* u = const_cast<double*>(b.in);
            stage_tile<PH, W3, true>(g, tl, it.i1_0, b.g[dir] - 2, 0, u, u, b.uh, pp, first, dtodx, spar->ch, fc,
                                     smem, status, true, true);
        } else {
            const long long n = (long long)(it.end - it.beg) * NV;
            for (long long t = threadIdx.x; t < n; t += blockDim.x) {
                const int slot = it.beg + (int)(t / NV);
                const int v = (int)(t % NV);
                double acc = 0.0;
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int sfine = ra.src[4 * slot + q];
                    if (sfine >= 0) acc = acc + __ldcg(ra.out_flux + (long long)sfine * NV + v);
                }
                ra.in_flux[(long long)slot * NV + v] = ra.scale * acc;
            }
        }
        if (it.fence) __threadfence();                     // this CTA's writes before its count
        __syncthreads();
        if (threadIdx.x == 0) atomicAdd(counters + 1 + (it.kind == 0 ? 0 : ra.nlev) + it.level, 1u);
    }
    flush_status(status, gstatus);
}

// -------------------------------------------------------------------------
// The unsplit scheme (RIEMANN_UNSPLIT, src/scheme/unsplit_schemes).
// -------------------------------------------------------------------------

// Face fluxes of one direction (solve_cg_unsplit.F90:95-138,
// unsplit_mag_modules.F90:56-128): the pencils through the interior, whole or
// in chunks with a 2-cell halo as k_stage; the flux through the face between
// storage cells s and s+1 goes to F at cell s+1 (pflux(:, i) is the flux
// through cell i's left face), in the state's own plane order.
template <class PH, int MAXT, bool W3 = false, bool FC = false>
__global__ void __launch_bounds__(MAXT, 2) k_unsplit_flux(Geom g, Tile tl, const double* __restrict__ uin,
                                                      double* __restrict__ F, PhysParams pp,
                                                      const StepParams* __restrict__ spar,
                                                      unsigned* __restrict__ gstatus, FcArgs fc = FcArgs{})
{
    extern __shared__ double smem[];
    constexpr int NV = PH::NV;
    const int P = tl.P, T = tl.T, PT = P * T;
    const Smem sm{smem, smem + NV * PT, smem + 2 * NV * PT, PT};
    const int tid = threadIdx.x;
    int p, t;
    if (tl.xfast) { t = tid % T; p = tid / T; }
    else { p = tid % P; t = tid / P; }
    const int spp = tl.xfast ? T : 1, st = tl.xfast ? 1 : P;
    const int me = p * spp + t * st;
    const int i1 = blockIdx.x * P + p;
    const int c0 = blockIdx.y * tl.L;
    const int i2 = blockIdx.z;
    const int n = g.ext_d;
    const int s = c0 - tl.halo + t;
    const bool valid = (tid < PT) && (i1 < g.n1) && s >= 0 && s < n;
    const bool own = valid && s >= c0 && s < c0 + tl.L;
    const long long off = (long long)s * g.sd + (long long)(g.g1 + i1) * g.s1 + (long long)(g.g2 + i2) * g.s2;
    double w[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) w[v] = 0.0;
    if (valid) load_cell<PH>(uin, off, g, w);
    Roles r;
    r.q = valid;
    r.end = (s == 0) ? -1 : ((s == n - 1) ? 1 : 0);
    r.slope = valid && (r.end != 0 || (t >= 1 && t <= T - 2));
    const bool next_slope = (s + 1 < n) && (t + 1 <= T - 1) && ((s + 1 == n - 1) || (t + 1 <= T - 2));
    r.flux = r.slope && next_slope;
    r.upd = false;
    r.keep = false;
    unsigned status = 0;
    const double* fc_in = nullptr;
    double* fc_out = nullptr;
    if constexpr (FC)
        if (valid) fc_slots<PH>(fc, g, i1, i2, s, fc_in, fc_out);
    rk_stage<PH, false, W3, FC>(sm, me, me - st, me + st, r, w, uin, uin, off, g, 0.0, spar->ch, pp, status, nullptr,
                                fc_in, fc_out);
    if (own && r.flux) {
        double f[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) f[v] = sm.Q[v * PT + me];
        store_cell<PH>(F, off + g.sd, g, f);
    }
}

}  // namespace pk
