// pk_adjoint_kernels.cuh -- the adjoint of one fused directional sweep.
//
// Forward map of a sweep on a periodic block (the fused kernel):
//   U*  = floors1(U  + c1 D(U)),   c1 = (dt/2)/dl      (RK2_1)
//   U'' = floors2(U  + c2 D(U*)),  c2 =  dt   /dl      (RK2_2), psi'' *= fac
// with D(V)_i = F_{i-1/2}(V) - F_{i+1/2}(V).  Given lam'' = dL/dU'' the kernel
// returns dL/dU:
//   mu2  = floors2^T (fac-scaled lam'')
//   lam  = mu2 + floors1^T( c2 D'(U*)^T mu2 ) + c1 D'(U)^T floors1^T(...)
// Each CTA recomputes both forward stages for its tile (8-cell halo read with
// periodic wrap), recording which floors clipped, then runs the two
// transposed divergences back to front.  D'(V)^T mu is assembled face by
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
// computed (cells [max(va+3, ma+2), min(vb-3, mb-2)) ).
template <class PH>
PK_DEV void adj_divergence(const AdjSmem& sm, int me, int st, int t, bool active, int va, int vb, int ma, int mb,
                           const double (&V)[PH::NV], const double (&mu)[PH::NV], double ch, const PhysParams& pp,
                           double (&out)[PH::NV])
{
    constexpr int NV = PH::NV;
    const int PT = sm.PT;
    auto qv = [&](int x) { return active && x >= va && x < vb; };
    auto sv = [&](int x) { return active && x > va && x < vb - 1; };
    auto mv = [&](int x) { return active && x >= ma && x < mb; };
    auto fv = [&](int x) { return sv(x) && sv(x + 1) && mv(x) && mv(x + 1); };   // face x+1/2
    // A: primitives and mu
    if (qv(t)) {
        double q[NV];
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
            const double s = slope_interior(lim, qc - sm.Q[v * PT + me - st], sm.Q[v * PT + me + st] - qc);
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
            qr[v] = sm.R[v * PT + me + st];
            fb[v] = sm.M[v * PT + me + st] - sm.M[v * PT + me];
        }
        riemann_adj<PH>(ql, qr, ch, pp, fb, gl, gr);
#pragma unroll
        for (int v = 0; v < NV; ++v) sm.R[v * PT + me + st] = gr[v];
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
            slope_adj(lim, qc - sm.Q[v * PT + me - st], sm.Q[v * PT + me + st] - qc, 0.5 * gl[v] - 0.5 * grr, dlb, drb);
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
            if (sp) x -= sm.L[v * PT + me + st];
            if (sn) x += sm.M[v * PT + me - st];
            qb[v] = x;
        }
        utoq_adj<PH>(V, qb, out, pp);
    }
    __syncthreads();
}

// Adjoint of one fused sweep (k_sweep_fused) of a periodic block:
// lam_out = dL/d(sweep output) in, lam_in = dL/d(sweep input) out.
// grid: x = ortho-1 tiles of P pencils, y = chunks of L cells, z = ortho-2;
// each tile spans L + 16 cells (8-cell halo) along the sweep.
template <class PH, int MAXT, int MINB>
__global__ void __launch_bounds__(MAXT, MINB) k_sweep_adj(Geom g, Tile tl, const double* __restrict__ uin,
                                                         const double* __restrict__ lam_out,
                                                         double* __restrict__ lam_in, PhysParams pp, double dl,
                                                         const StepParams* __restrict__ sp, int apply_fac,
                                                         unsigned* __restrict__ gstatus)
{
    extern __shared__ double smem[];
    constexpr int NV = PH::NV;
    const int P = tl.P, T = tl.T, PT = P * T;
    const Smem fsm{smem, smem + NV * PT, smem + 2 * NV * PT, PT};
    const AdjSmem asm_{smem, smem + NV * PT, smem + 2 * NV * PT, smem + 3 * NV * PT, PT};
    const int tid = threadIdx.x;
    int p, t;
    if (tl.xfast) { t = tid % T; p = tid / T; }
    else { p = tid % P; t = tid / P; }
    const int spp = tl.xfast ? T : 1, st = tl.xfast ? 1 : P;
    const int me = p * spp + t * st;
    const int i1 = blockIdx.x * P + p;
    const int c0 = blockIdx.y * tl.L;
    const int i2 = blockIdx.z;
    const bool active = (tid < PT) && (i1 < g.n1);
    const int s = c0 - 8 + t;
    const long long off = (long long)(g.g_d + wrap(s, g.n_d)) * g.sd + (long long)(g.g1 + i1) * g.s1 +
                          (long long)(g.g2 + i2) * g.s2;
    const double dt = sp->dt, ch = sp->ch, fac = apply_fac ? sp->psi_fac : 1.0;
    const double c1 = (0.5 * dt) / dl, c2 = (1.0 * dt) / dl;
    unsigned status = 0;
    double w[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) w[v] = 0.0;
    if (active) load_cell<PH>(uin, off, g, w);
    // forward stage 1 on [0, T) -> U* on [2, T-2)
    FloorRec rec1{0, 0}, rec2{0, 0};
    Roles r;
    r.end = 0;
    r.keep = false;
    r.q = active;
    r.slope = active && t >= 1 && t < T - 1;
    r.flux = active && t >= 1 && t < T - 2;
    r.upd = active && t >= 2 && t < T - 2;
    rk_stage<PH, true>(fsm, me, st, r, w, uin, uin, off, g, c1, ch, pp, status, &rec1);
    double us[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) us[v] = w[v];
    // forward stage 2 on [2, T-2) -> U'' on [4, T-4)
    r.q = active && t >= 2 && t < T - 2;
    r.slope = active && t >= 3 && t < T - 3;
    r.flux = active && t >= 3 && t < T - 4;
    r.upd = active && t >= 4 && t < T - 4;
    rk_stage<PH, true>(fsm, me, st, r, w, uin, uin, off, g, c2, ch, pp, status, &rec2);
    // adjoint of the stage-2 floors (and of the psi damping folded into this sweep)
    double lam[NV], mu[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) lam[v] = mu[v] = 0.0;
    if (active && t >= 4 && t < T - 4) {
        load_cell<PH>(lam_out, off, g, mu);
        if (PH::MHD) mu[PH::IB + 3] = mu[PH::IB + 3] * fac;
        floors_adj<PH>(w, rec2, mu);
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            lam[v] = mu[v];
            mu[v] = c2 * mu[v];
        }
    }
    // c2 D'(U*)^T mu2 -> valid on [6, T-6)
    double rho[NV];
    adj_divergence<PH>(asm_, me, st, t, active, 2, T - 2, 4, T - 4, us, mu, ch, pp, rho);
    // adjoint of the stage-1 floors
#pragma unroll
    for (int v = 0; v < NV; ++v) mu[v] = 0.0;
    if (active && t >= 6 && t < T - 6) {
#pragma unroll
        for (int v = 0; v < NV; ++v) mu[v] = rho[v];
        floors_adj<PH>(us, rec1, mu);
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            lam[v] += mu[v];
            mu[v] = c1 * mu[v];
        }
    }
    // c1 D'(U)^T mu1 -> valid on [8, T-8)
    if (active) load_cell<PH>(uin, off, g, w);
    adj_divergence<PH>(asm_, me, st, t, active, 0, T, 6, T - 6, w, mu, ch, pp, rho);
    if (active && t >= 8 && t < T - 8 && s < c0 + tl.L && s < g.n_d) {
#pragma unroll
        for (int v = 0; v < NV; ++v) lam[v] += rho[v];
        store_cell<PH>(lam_in, off, g, lam);
    }
    flush_status(status, gstatus);
}

}  // namespace pk
