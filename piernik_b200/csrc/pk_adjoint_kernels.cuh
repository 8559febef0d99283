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

}  // namespace pk
