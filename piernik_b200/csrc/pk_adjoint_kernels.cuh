// pk_adjoint_kernels.cuh -- the adjoint of one fused directional sweep.
//
// Forward map of a sweep on a periodic block (the fused kernel):
//   U*  = floors1(U  + c1 D(U)),   c1 = (dt/2)/dl      (RK2_1)
//   U'' = floors2(U  + c2 D(U*)),  c2 =  dt   /dl      (RK2_2), psi'' *= fac
// with D(V)_i = F_{i-1/2}(V) - F_{i+1/2}(V).  Given lam'' = dL/dU'' the kernel
// returns dL/dU:
//   mu2  = floors2^T (fac-scaled lam'')
//   lam  = mu2 + floors1^T( c2 D'(U*)^T mu2 ) + c1 D'(U)^T floors1^T(...)
// The backward pass runs it as three kernels per sweep:
//   k_sweep_fused_rec  the forward sweep again, also storing U* and which
//                      floors clipped in either stage (2 bytes per cell);
//   k_adj_stage2       mu2, rho = c2 D'(U*)^T mu2, mu1 = floors1^T rho:
//                      writes lam_acc = mu2 + mu1 and m1 = c1 mu1;
//   k_adj_stage1       lam = lam_acc + D'(U)^T m1.
// Each adjoint kernel holds one transposed divergence (one Riemann adjoint per
// face, no forward Riemann solve) over a tile with a 3-cell halo read with
// periodic wrap.  D'(V)^T mu is assembled face by
// face: g_{k+1/2} = mu_{k+1} - mu_k, the Riemann adjoint gives the adjoints of
// the two face states, the slope adjoint spreads them over the 3-cell
// stencil, and utoq's adjoint maps primitive adjoints to conservative ones.
#pragma once
#include "pk_adjoint.cuh"
#include "pk_kernels.cuh"
#include "pk_staged.cuh"

namespace pk {

struct AdjSmem {
    double* Q;   // primitives, then the dl adjoint of each slope
    double* L;   // left state of the right face, then the dl adjoint of the slope
    double* R;   // right state of the left face, then the right-state adjoint of the left face
    double* M;   // mu, then the dr adjoint of the slope
    int PT;
};

// out = D'(V)^T mu for the tile: V valid on tile cells [va, vb), mu valid on
// [ma, mb); out is exact where every face whose stencil holds the cell was
// computed (cells [max(va+3, ma+2), min(vb-3, mb-2)) ).  mp / mn: the slots
// of the previous / next cell along the pencil; circ: the tile is a whole
// periodic pencil (every cell valid, neighbours wrap).
// The cell's V is read from vsrc (at off, swept order) in phase A and again
// in phase E, not held in registers across the Riemann adjoint of phase C,
// which needs every register it can get.
template <class PH>
PK_DEV void adj_divergence(const AdjSmem& sm, int me, int mp, int mn, bool circ, int t, bool active, int va, int vb,
                           int ma, int mb, const double* vsrc, long long off, const Geom& g,
                           const double (&mu)[PH::NV], double ch, const PhysParams& pp, double (&out)[PH::NV])
{
    constexpr int NV = PH::NV;
    const int PT = sm.PT;
    auto qv = [&](int x) { return active && (circ || (x >= va && x < vb)); };
    auto sv = [&](int x) { return active && (circ || (x > va && x < vb - 1)); };
    auto mv = [&](int x) { return active && (circ || (x >= ma && x < mb)); };
    auto fv = [&](int x) { return sv(x) && sv(x + 1) && mv(x) && mv(x + 1); };   // face x+1/2
    // A: primitives and mu
    if (qv(t)) {
        double V[NV], q[NV];
        load_cell<PH>(vsrc, off, g, V);
        utoq<PH>(V, q, pp);
#pragma unroll
        for (int v = 0; v < NV; ++v) sm.Q[v * PT + me] = q[v];
    }
    if (mv(t)) {
#pragma unroll
        for (int v = 0; v < NV; ++v) sm.M[v * PT + me] = mu[v];
    }
    __syncthreads();
    // B: face states of the primal reconstruction
    if (sv(t)) {
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            const int lim = (PH::MHD && v >= PH::IB) ? pp.limb : pp.lim;
            const double qc = sm.Q[v * PT + me];
            const double s = slope_interior(lim, qc - sm.Q[v * PT + mp], sm.Q[v * PT + mn] - qc);
            const double dqh = 0.5 * s;
            sm.L[v * PT + me] = qc + dqh;
            sm.R[v * PT + me] = qc - dqh;
        }
    }
    __syncthreads();
    // C: Riemann adjoint of the right face: gl stays here, gr goes to the right neighbour's R slot
    double gl[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) gl[v] = 0.0;
    if (fv(t)) {
        double ql[NV], qr[NV], fb[NV], gr[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            ql[v] = sm.L[v * PT + me];
            qr[v] = sm.R[v * PT + mn];
            fb[v] = sm.M[v * PT + mn] - sm.M[v * PT + me];
        }
        riemann_adj<PH>(ql, qr, ch, pp, fb, gl, gr);
#pragma unroll
        for (int v = 0; v < NV; ++v) sm.R[v * PT + mn] = gr[v];
    }
    __syncthreads();
    // D: primitive adjoint of the cell itself and the slope adjoint
    double qb[NV];
    const bool prev = fv(t - 1);
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        const double grr = prev ? sm.R[v * PT + me] : 0.0;
        qb[v] = gl[v] + grr;
        if (sv(t)) {
            const int lim = (PH::MHD && v >= PH::IB) ? pp.limb : pp.lim;
            const double qc = sm.Q[v * PT + me];
            double dlb, drb;
            slope_adj(lim, qc - sm.Q[v * PT + mp], sm.Q[v * PT + mn] - qc, 0.5 * gl[v] - 0.5 * grr, dlb, drb);
            sm.L[v * PT + me] = dlb;
            sm.M[v * PT + me] = drb;
        }
    }
    __syncthreads();
    // E: gather the slope adjoints of the 3-cell stencil, then utoq's adjoint
#pragma unroll
    for (int v = 0; v < NV; ++v) out[v] = 0.0;
    if (qv(t)) {
        const bool s0 = sv(t), sp = sv(t + 1), sn = sv(t - 1);
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            double x = qb[v];
            if (s0) x += sm.L[v * PT + me] - sm.M[v * PT + me];
            if (sp) x -= sm.L[v * PT + mn];
            if (sn) x += sm.M[v * PT + mp];
            qb[v] = x;
        }
        double V[NV];
        load_cell<PH>(vsrc, off, g, V);
        utoq_adj<PH>(V, qb, out, pp);
    }
    __syncthreads();
}

PK_DEV FloorRec unpack_floors(unsigned short f, int stage)
{
    const int sh = stage == 1 ? 0 : 6;
    return FloorRec{(unsigned)(f >> sh) & 7u, (unsigned)(f >> (sh + 3)) & 7u};
}

// The fused forward sweep (k_sweep_fused) that also stores the stage-1 state
// U* and the floor records of the owned cells: the backward pass's segment
// recomputation.
template <class PH, int MAXT, int MINB>
__global__ void __launch_bounds__(MAXT, MINB) k_sweep_fused_rec(Geom g, Tile tl, const double* __restrict__ uin,
                                                               double* __restrict__ uout, double* __restrict__ ustar,
                                                               unsigned short* __restrict__ flags, PhysParams pp,
                                                               double dl, const StepParams* __restrict__ sp,
                                                               int apply_fac, unsigned* __restrict__ gstatus)
{
    extern __shared__ double smem[];
    unsigned status = 0;
    fused_tile<PH, true>(g, tl, blockIdx.x * tl.P, blockIdx.y * tl.L, blockIdx.z, uin, uout, pp, sp, dl, apply_fac, smem,
                         status, ustar, flags);
    flush_status(status, gstatus);
}

// Tile position shared by the two adjoint kernels: 3-cell halo.
struct AdjPos {
    int t, me, mp, mn, s;
    int seg;                // instance of the tile (cells stacked along z), for the step scalars
    bool active, own, circ;
    long long off;
};

PK_DEV AdjPos adj_pos(const Geom& g, const Tile& tl)
{
    AdjPos a;
    const int P = tl.P, T = tl.T, PT = P * T;
    const int tid = threadIdx.x;
    int p;
    if (tl.xfast) { a.t = tid % T; p = tid / T; }
    else { p = tid % P; a.t = tid / P; }
    const int spp = tl.xfast ? T : 1;
    const int st = tl.xfast ? 1 : P;
    a.me = p * spp + a.t * st;
    a.circ = tl.circ;
    a.mp = a.circ ? p * spp + (a.t == 0 ? T - 1 : a.t - 1) * st : a.me - st;
    a.mn = a.circ ? p * spp + (a.t == T - 1 ? 0 : a.t + 1) * st : a.me + st;
    const int i1 = blockIdx.x * P + p;
    const int c0 = blockIdx.y * tl.L;
    a.active = (tid < PT) && (i1 < g.n1);
    a.s = a.circ ? c0 + a.t : c0 - 3 + a.t;
    a.seg = g.seg_len ? ((g.seg_along ? c0 : (int)blockIdx.z) / g.seg_len) : 0;
    a.own = a.active && (a.circ || (a.t >= 3 && a.t < T - 3 && a.s < c0 + tl.L && a.s < g.n_d));
    a.off = (long long)(g.g_d + wrap(a.s, g.n_d)) * g.sd + (long long)(g.g1 + i1) * g.s1 +
            (long long)(g.g2 + blockIdx.z) * g.s2;
    return a;
}

// Stage-2 half of the sweep adjoint.  In: U* (ustar), the sweep output U''
// (read only where an energy floor clipped), floor records, lam'' (lam_out).
// Out on every interior cell: lam_acc = mu2 + mu1 and m1 = c1 mu1.
template <class PH, int MAXT, int MINB>
__global__ void __launch_bounds__(MAXT, MINB) k_adj_stage2(Geom g, Tile tl, const double* __restrict__ ustar,
                                                          const double* __restrict__ uout,
                                                          const unsigned short* __restrict__ flags,
                                                          const double* __restrict__ lam_out,
                                                          double* __restrict__ lam_acc, double* __restrict__ m1,
                                                          PhysParams pp, double dl, const StepParams* __restrict__ sp,
                                                          int apply_fac)
{
    extern __shared__ double smem[];
    constexpr int NV = PH::NV;
    const int PT = tl.P * tl.T;
    const AdjSmem asm_{smem, smem + NV * PT, smem + 2 * NV * PT, smem + 3 * NV * PT, PT};
    const AdjPos a = adj_pos(g, tl);
    const StepParams stp = sp[a.seg];
    const double dt = stp.dt, ch = stp.ch, fac = apply_fac ? stp.psi_fac : 1.0;
    const double c1 = (0.5 * dt) / dl, c2 = (1.0 * dt) / dl;
    // mu2 = floors2^T (fac-scaled lam''); formed before the divergence and
    // again after it rather than kept in registers across it
    auto mu2_of = [&](double (&m)[NV]) {
        load_cell<PH>(lam_out, a.off, g, m);
        if (PH::MHD) m[PH::IB + 3] = m[PH::IB + 3] * fac;
        const FloorRec r2 = unpack_floors(flags[a.off], 2);
        if (r2.en || r2.dn) {
            double w[NV];
            load_cell<PH>(uout, a.off, g, w);
            floors_adj<PH>(w, r2, m);
        }
    };
    double mu[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) mu[v] = 0.0;
    if (a.active) {
        mu2_of(mu);
#pragma unroll
        for (int v = 0; v < NV; ++v) mu[v] = c2 * mu[v];
    }
    double rho[NV];
    adj_divergence<PH>(asm_, a.me, a.mp, a.mn, a.circ, a.t, a.active, 0, tl.T, 0, tl.T, ustar, a.off, g, mu, ch, pp,
                       rho);
    if (a.own) {
        double V[NV], mu2[NV];
        load_cell<PH>(ustar, a.off, g, V);
        floors_adj<PH>(V, unpack_floors(flags[a.off], 1), rho);
        mu2_of(mu2);
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            mu2[v] += rho[v];
            rho[v] = c1 * rho[v];
        }
        store_cell<PH>(lam_acc, a.off, g, mu2);
        store_cell<PH>(m1, a.off, g, rho);
    }
}

// Stage-1 half: lam_io = lam_acc + D'(U)^T m1, in place.
template <class PH, int MAXT, int MINB>
__global__ void __launch_bounds__(MAXT, MINB) k_adj_stage1(Geom g, Tile tl, const double* __restrict__ uin,
                                                          const double* __restrict__ m1, double* __restrict__ lam_io,
                                                          PhysParams pp, const StepParams* __restrict__ sp)
{
    extern __shared__ double smem[];
    constexpr int NV = PH::NV;
    const int PT = tl.P * tl.T;
    const AdjSmem asm_{smem, smem + NV * PT, smem + 2 * NV * PT, smem + 3 * NV * PT, PT};
    const AdjPos a = adj_pos(g, tl);
    double mu[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) mu[v] = 0.0;
    if (a.active) load_cell<PH>(m1, a.off, g, mu);
    double rho[NV];
    adj_divergence<PH>(asm_, a.me, a.mp, a.mn, a.circ, a.t, a.active, 0, tl.T, 0, tl.T, uin, a.off, g, mu, sp[a.seg].ch,
                       pp, rho);
    if (a.own) {
        double l[NV];
        load_cell<PH>(lam_io, a.off, g, l);
#pragma unroll
        for (int v = 0; v < NV; ++v) l[v] += rho[v];
        store_cell<PH>(lam_io, a.off, g, l);
    }
}

// ---------------------------------------------------------------------------
// TMA-staged whole-pencil adjoint kernels.  As in k_sweep_staged a tile is two
// neighbouring pencils, whole along the sweep (n <= 256, periodic, no halo),
// run one after the other through the same per-cell code as k_adj_stage2 /
// k_adj_stage1 (adj_divergence over a circular tile) with the inputs read from
// shared-memory boxes [2 pencils x n cells x NV planes] (a Geom whose plane
// stride is the box's 2n).  The kernels are persistent, one 256-thread CTA per
// SM (the Riemann adjoint takes 255 registers) walking the tiles with stride
// gridDim.x, and the input boxes are double-buffered: thread 0 issues the
// cp.async.bulk.tensor loads of the next tile into the other buffer while the
// CTA computes the current one, so the gather of the y/z boxes' 16-byte rows
// is not waited for.  Each buffer has its own mbarrier (bounded waits:
// PK_ST_TIMEOUT after 2^24 polls).  Results equal the tiled kernels' bit for
// bit.
// ---------------------------------------------------------------------------

PK_DEV void adj_bars_init(unsigned long long* bars)
{
    if (threadIdx.x == 0) {
        mbar_init(bars, 1);
        mbar_init(bars + 1, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        fence_proxy_async();
    }
    __syncthreads();
}

// bounded wait for phase `parity` of bar; false (for every thread) if it gave up
PK_DEV bool adj_bar_wait(unsigned long long* bar, unsigned parity)
{
    bool ready = false;
    for (int it = 0; it < (1 << 24) && !ready; ++it) ready = mbar_try_wait(bar, parity);
    return __syncthreads_and(ready) != 0;
}

// doubles per box, rounded up to 128 bytes (each box starts 128-byte aligned)
PK_PHYS int adj_box_doubles(int nv, int n) { return (2 * nv * n + 15) / 16 * 16; }

// tile tau: pencil pair (2 * (tau % npair), +1) along ortho-1 at ortho-2 index
// tau / npair; c = the box's tensor coordinates (x, y, z, plane)
PK_DEV void adj_tile(const Geom& g, int dir, int tau, int npair, int& i1_0, int& i2, int (&c)[4])
{
    i1_0 = 2 * (tau % npair);
    i2 = tau / npair;
    const int o1 = dir == 0 ? 1 : 0, o2 = dir == 2 ? 1 : 2;
    c[dir] = g.g_d;
    c[o1] = g.g1 + i1_0;
    c[o2] = g.g2 + i2;
    c[3] = 0;
}

// Stage 2.  Buffer b holds the boxes U* (then m1) and lam'' (then lam_acc);
// each cell's results go into the box slots only it read and TMA stores write
// both boxes out; the next tile's loads into the other buffer wait for the
// previous tile's stores to have read it (issued between the two pencils).
// Shared memory: 2 buffers x 2 boxes of 2 NV n doubles (each rounded up to
// 128 bytes), the four planes of the tile (4 NV n), two mbarriers.
template <class PH>
__global__ void __launch_bounds__(256, 1) k_adj_staged2(const __grid_constant__ CUtensorMap t_ustar,
                                                        const __grid_constant__ CUtensorMap t_lamout,
                                                        const __grid_constant__ CUtensorMap t_lamacc,
                                                        const __grid_constant__ CUtensorMap t_m1, Geom g,
                                                        const double* __restrict__ uout,
                                                        const unsigned short* __restrict__ flags, PhysParams pp,
                                                        double dl, const StepParams* __restrict__ sp, int apply_fac,
                                                        int dir, unsigned* __restrict__ gstatus)
{
    constexpr int NV = PH::NV;
    extern __shared__ __align__(128) double smem[];
    const int n = g.n_d;
    const int bd = adj_box_doubles(NV, n);
    double* pl = smem + 4 * bd;
    const AdjSmem asm_{pl, pl + NV * n, pl + 2 * NV * n, pl + 3 * NV * n, n};
    unsigned long long* bars = reinterpret_cast<unsigned long long*>(pl + 4 * NV * n);
    const int npair = (g.n1 + 1) / 2, ntiles = npair * g.n2, G = (int)gridDim.x;
    const unsigned bytes = (unsigned)(2 * (2 * NV * n * sizeof(double)));
    auto issue = [&](int tau, int b) {                   // thread 0: the tile's input boxes into buffer b
        int i1, j2, c[4];
        adj_tile(g, dir, tau, npair, i1, j2, c);
        mbar_expect_tx(bars + b, bytes);
        tma_load_4d(smem + 2 * b * bd, &t_ustar, c[0], c[1], c[2], c[3], bars + b);
        tma_load_4d(smem + (2 * b + 1) * bd, &t_lamout, c[0], c[1], c[2], c[3], bars + b);
    };
    adj_bars_init(bars);
    if (threadIdx.x == 0 && (int)blockIdx.x < ntiles) issue(blockIdx.x, 0);
    Geom gb = g;                                         // the boxes as component planes of 2n cells
    gb.plane = 2 * n;
    const int st_t = dir == 0 ? 1 : 2, st_p = dir == 0 ? n : 1;
    const int t = threadIdx.x;
    const int mp = t == 0 ? n - 1 : t - 1, mn = t == n - 1 ? 0 : t + 1;
    int k = 0;
    for (int tau = blockIdx.x; tau < ntiles; tau += G, ++k) {
        const int b = k & 1;
        if (!adj_bar_wait(bars + b, (unsigned)((k >> 1) & 1))) {
            if (threadIdx.x == 0) {
                atomicOr(gstatus, ST_TIMEOUT);
                asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
            }
            return;
        }
        double* bv = smem + 2 * b * bd;                  // U*, then m1
        double* bl = bv + bd;                            // lam'', then lam_acc
        int i1_0, i2, c[4];
        adj_tile(g, dir, tau, npair, i1_0, i2, c);
        const StepParams stp = sp[g.seg_len ? i2 / g.seg_len : 0];   // stacked instances: this tile's
        const double dt = stp.dt, ch = stp.ch, fac = apply_fac ? stp.psi_fac : 1.0;
        const double c1 = (0.5 * dt) / dl, c2 = (1.0 * dt) / dl;
#pragma unroll 1
        for (int p = 0; p < 2; ++p) {
            if (p == 1 && threadIdx.x == 0 && tau + G < ntiles) {
                // the other buffer held the previous tile: its stores must have read it
                asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
                issue(tau + G, b ^ 1);
            }
            if (i1_0 + p >= g.n1) break;                 // the same for the whole CTA
            const bool active = t < n;
            const int slot = active ? t * st_t + p * st_p : 0;
            const long long goff = (long long)(g.g_d + (active ? t : 0)) * g.sd +
                                   (long long)(g.g1 + i1_0 + p) * g.s1 + (long long)(g.g2 + i2) * g.s2;
            const unsigned short fl = active ? flags[goff] : (unsigned short)0;
            auto mu2_of = [&](double (&m)[NV]) {
                load_cell<PH>(bl, slot, gb, m);
                if (PH::MHD) m[PH::IB + 3] = m[PH::IB + 3] * fac;
                const FloorRec r2 = unpack_floors(fl, 2);
                if (r2.en || r2.dn) {
                    double w[NV];
                    load_cell<PH>(uout, goff, g, w);
                    floors_adj<PH>(w, r2, m);
                }
            };
            double mu[NV];
#pragma unroll
            for (int v = 0; v < NV; ++v) mu[v] = 0.0;
            if (active) {
                mu2_of(mu);
#pragma unroll
                for (int v = 0; v < NV; ++v) mu[v] = c2 * mu[v];
            }
            double rho[NV];
            adj_divergence<PH>(asm_, t, mp, mn, true, t, active, 0, n, 0, n, bv, slot, gb, mu, ch, pp, rho);
            if (active) {
                double V[NV], mu2[NV];
                load_cell<PH>(bv, slot, gb, V);
                floors_adj<PH>(V, unpack_floors(fl, 1), rho);
                mu2_of(mu2);
#pragma unroll
                for (int v = 0; v < NV; ++v) {
                    mu2[v] += rho[v];
                    rho[v] = c1 * rho[v];
                }
                store_cell<PH>(bl, slot, gb, mu2);
                store_cell<PH>(bv, slot, gb, rho);
            }
        }
        fence_proxy_async();
        __syncthreads();
        if (threadIdx.x == 0) {
            tma_store_4d(&t_lamacc, bl, c[0], c[1], c[2], c[3]);
            tma_store_4d(&t_m1, bv, c[0], c[1], c[2], c[3]);
        }
    }
    if (threadIdx.x == 0) asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}

// Stage 1.  Buffer b holds the boxes U and m1 (inputs only); lam is updated in
// place with plain loads and stores at the cell's offset, so a buffer is free
// as soon as its tile is computed and the load of the tile after next goes
// into it at once.  Shared memory as stage 2.
template <class PH>
__global__ void __launch_bounds__(256, 1) k_adj_staged1(const __grid_constant__ CUtensorMap t_uin,
                                                        const __grid_constant__ CUtensorMap t_m1, Geom g,
                                                        double* __restrict__ lam, PhysParams pp,
                                                        const StepParams* __restrict__ sp, int dir,
                                                        unsigned* __restrict__ gstatus)
{
    constexpr int NV = PH::NV;
    extern __shared__ __align__(128) double smem[];
    const int n = g.n_d;
    const int bd = adj_box_doubles(NV, n);
    double* pl = smem + 4 * bd;
    const AdjSmem asm_{pl, pl + NV * n, pl + 2 * NV * n, pl + 3 * NV * n, n};
    unsigned long long* bars = reinterpret_cast<unsigned long long*>(pl + 4 * NV * n);
    const int npair = (g.n1 + 1) / 2, ntiles = npair * g.n2, G = (int)gridDim.x;
    const unsigned bytes = (unsigned)(2 * (2 * NV * n * sizeof(double)));
    auto issue = [&](int tau, int b) {
        int i1, j2, c[4];
        adj_tile(g, dir, tau, npair, i1, j2, c);
        mbar_expect_tx(bars + b, bytes);
        tma_load_4d(smem + 2 * b * bd, &t_uin, c[0], c[1], c[2], c[3], bars + b);
        tma_load_4d(smem + (2 * b + 1) * bd, &t_m1, c[0], c[1], c[2], c[3], bars + b);
    };
    adj_bars_init(bars);
    if (threadIdx.x == 0) {
        if ((int)blockIdx.x < ntiles) issue(blockIdx.x, 0);
        if ((int)blockIdx.x + G < ntiles) issue(blockIdx.x + G, 1);
    }
    Geom gb = g;
    gb.plane = 2 * n;
    const int st_t = dir == 0 ? 1 : 2, st_p = dir == 0 ? n : 1;
    const int t = threadIdx.x;
    const int mp = t == 0 ? n - 1 : t - 1, mn = t == n - 1 ? 0 : t + 1;
    int k = 0;
    for (int tau = blockIdx.x; tau < ntiles; tau += G, ++k) {
        const int b = k & 1;
        if (!adj_bar_wait(bars + b, (unsigned)((k >> 1) & 1))) {
            if (threadIdx.x == 0) {
                atomicOr(gstatus, ST_TIMEOUT);
                // the other buffer's load (the next tile) may still be in
                // flight: let it land (bounded) before the CTA's memory goes
                if (tau + G < ntiles) {
                    bool done = false;
                    for (int it = 0; it < (1 << 24) && !done; ++it)
                        done = mbar_try_wait(bars + (b ^ 1), (unsigned)(((k + 1) >> 1) & 1));
                }
            }
            return;
        }
        const double* bv = smem + 2 * b * bd;            // U
        const double* bm = bv + bd;                      // m1
        int i1_0, i2, c[4];
        adj_tile(g, dir, tau, npair, i1_0, i2, c);
        const double ch = sp[g.seg_len ? i2 / g.seg_len : 0].ch;
#pragma unroll 1
        for (int p = 0; p < 2; ++p) {
            if (i1_0 + p >= g.n1) break;
            const bool active = t < n;
            const int slot = active ? t * st_t + p * st_p : 0;
            const long long goff = (long long)(g.g_d + (active ? t : 0)) * g.sd +
                                   (long long)(g.g1 + i1_0 + p) * g.s1 + (long long)(g.g2 + i2) * g.s2;
            double mu[NV];
#pragma unroll
            for (int v = 0; v < NV; ++v) mu[v] = 0.0;
            if (active) load_cell<PH>(bm, slot, gb, mu);
            double rho[NV];
            adj_divergence<PH>(asm_, t, mp, mn, true, t, active, 0, n, 0, n, bv, slot, gb, mu, ch, pp, rho);
            if (active) {
                double l[NV];
                load_cell<PH>(lam, goff, g, l);
#pragma unroll
                for (int v = 0; v < NV; ++v) l[v] += rho[v];
                store_cell<PH>(lam, goff, g, l);
            }
        }
        __syncthreads();                                 // every thread is done with buffer b
        if (threadIdx.x == 0 && tau + 2 * G < ntiles) {
            fence_proxy_async();
            issue(tau + 2 * G, b);
        }
    }
}

// Stage 1 with lam staged too, one tile per CTA (grid: x = pairs of pencils,
// z = ortho-2): the boxes U, m1 and lam are loaded together, lam is updated in
// its box and written back by a TMA store.  Used along y and z, where the
// persistent kernel's plain lam accesses would touch one 8-byte row fragment
// per thread; along x those accesses are contiguous and the persistent kernel
// is faster.  Shared memory: three boxes, the four planes, one mbarrier.
template <class PH>
__global__ void __launch_bounds__(256, 1) k_adj_staged1_boxed(const __grid_constant__ CUtensorMap t_uin,
                                                              const __grid_constant__ CUtensorMap t_m1,
                                                              const __grid_constant__ CUtensorMap t_lam, Geom g,
                                                              PhysParams pp, const StepParams* __restrict__ sp,
                                                              int dir, unsigned* __restrict__ gstatus)
{
    constexpr int NV = PH::NV;
    extern __shared__ __align__(128) double smem[];
    const int n = g.n_d;
    const int bd = adj_box_doubles(NV, n);
    double* bv = smem;                                   // U
    double* bm = smem + bd;                              // m1
    double* bl = smem + 2 * bd;                          // lam in, lam out
    double* pl = smem + 3 * bd;
    const AdjSmem asm_{pl, pl + NV * n, pl + 2 * NV * n, pl + 3 * NV * n, n};
    unsigned long long* bar = reinterpret_cast<unsigned long long*>(pl + 4 * NV * n);
    const int npair = (g.n1 + 1) / 2;
    int i1_0, i2, c[4];
    adj_tile(g, dir, (int)(blockIdx.z * npair + blockIdx.x), npair, i1_0, i2, c);
    adj_bars_init(bar);                                  // (initialises bar and bar + 1; only bar is used)
    if (threadIdx.x == 0) {
        mbar_expect_tx(bar, (unsigned)(3 * (2 * NV * n * sizeof(double))));
        tma_load_4d(bv, &t_uin, c[0], c[1], c[2], c[3], bar);
        tma_load_4d(bm, &t_m1, c[0], c[1], c[2], c[3], bar);
        tma_load_4d(bl, &t_lam, c[0], c[1], c[2], c[3], bar);
    }
    if (!adj_bar_wait(bar, 0)) {
        if (threadIdx.x == 0) atomicOr(gstatus, ST_TIMEOUT);
        return;
    }
    Geom gb = g;
    gb.plane = 2 * n;
    const int st_t = dir == 0 ? 1 : 2, st_p = dir == 0 ? n : 1;
    const double ch = sp[g.seg_len ? i2 / g.seg_len : 0].ch;
    const int t = threadIdx.x;
    const int mp = t == 0 ? n - 1 : t - 1, mn = t == n - 1 ? 0 : t + 1;
#pragma unroll 1
    for (int p = 0; p < 2; ++p) {
        if (i1_0 + p >= g.n1) break;
        const bool active = t < n;
        const int slot = active ? t * st_t + p * st_p : 0;
        double mu[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) mu[v] = 0.0;
        if (active) load_cell<PH>(bm, slot, gb, mu);
        double rho[NV];
        adj_divergence<PH>(asm_, t, mp, mn, true, t, active, 0, n, 0, n, bv, slot, gb, mu, ch, pp, rho);
        if (active) {
            double l[NV];
            load_cell<PH>(bl, slot, gb, l);
#pragma unroll
            for (int v = 0; v < NV; ++v) l[v] += rho[v];
            store_cell<PH>(bl, slot, gb, l);
        }
    }
    fence_proxy_async();
    __syncthreads();
    if (threadIdx.x == 0) {
        tma_store_4d(&t_lam, bl, c[0], c[1], c[2], c[3]);
        asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
    }
}

inline size_t adj_staged1_boxed_smem(int nv, int n)
{
    return ((size_t)3 * adj_box_doubles(nv, n) + (size_t)4 * nv * n) * sizeof(double) + 16;
}

// dynamic shared memory of the staged adjoint kernels (two buffers of two
// boxes, the four planes, two mbarriers) for nv planes and n cells
inline size_t adj_staged_smem(int nv, int n)
{
    return ((size_t)4 * adj_box_doubles(nv, n) + (size_t)4 * nv * n) * sizeof(double) + 16;
}

}  // namespace pk
