// pk_launch.cuh -- kernel launches for one physics configuration PH.  Each
// pk_phys_*.cu instantiates these for its PH, so the heavy kernels compile in
// parallel translation units.
#pragma once
#include <algorithm>

#include "pk_adjoint_kernels.cuh"
#include "pk_aux.cuh"
#include "pk_internal.h"
#include "pk_staged.cuh"

namespace pk {

template <class PH>
using FusedFn = void (*)(Geom, Tile, const double*, double*, PhysParams, double, const StepParams*, int, unsigned*);
template <class PH>
using BatchedFn = void (*)(const BlockDesc*, const WorkItem*, int, int, PhysParams, const StepParams*, int, unsigned*,
                           unsigned*);

// FAST: the tolerance-mode instantiations (pk_fast.cuh arithmetic), which only
// the pk_fast_*.cu units (compiled with contraction) may instantiate; every
// other unit instantiates FAST = false only, so that no kernel is compiled
// twice with different arithmetic
template <class PH, bool FAST = false>
FusedFn<PH> fused_variant(int v, bool w3 = false)
{
    if (w3) return k_sweep_fused<PH, 256, 2, true, FAST>;
    switch (v) {
    case 0: return k_sweep_fused<PH, 320, 1, false, FAST>;
    case 1: return k_sweep_fused<PH, 256, 1, false, FAST>;
    case 2: return k_sweep_fused<PH, 256, 2, false, FAST>;
    case 3: return k_sweep_fused<PH, 128, 3, false, FAST>;
    case 4: return k_sweep_fused<PH, 128, 4, false, FAST>;
    case 5: return k_sweep_fused<PH, 192, 2, false, FAST>;
    case 6: return k_sweep_fused<PH, 512, 1, false, FAST>;
    default: return k_sweep_fused<PH, 256, 2, false, FAST>;   // VAR_STAGED where the staged kernel cannot run
    }
}

template <class PH, bool FAST = false>
BatchedFn<PH> batched_variant(int v, bool w3 = false)
{
    if (w3) return k_sweep_batched<PH, 256, 2, true, FAST>;
    switch (v) {
    case 0: return k_sweep_batched<PH, 320, 1, false, FAST>;
    case 1: return k_sweep_batched<PH, 256, 1, false, FAST>;
    case 2: return k_sweep_batched<PH, 256, 2, false, FAST>;
    case 3: return k_sweep_batched<PH, 128, 3, false, FAST>;
    case 4: return k_sweep_batched<PH, 128, 4, false, FAST>;
    case 5: return k_sweep_batched<PH, 192, 2, false, FAST>;
    case 6: return k_sweep_batched<PH, 512, 1, false, FAST>;
    default: return k_sweep_batched<PH, 256, 2, false, FAST>;
    }
}

// dynamic shared memory limits of the fused and batched sweep kernels
template <class PH, bool FAST>
int set_fused_attr(pk_ctx* h)
{
    static bool done = false;
    if (!done) {
        for (int v = 0; v < NVARIANT; ++v) {
            PK_CUDA(h, cudaFuncSetAttribute(fused_variant<PH, FAST>(v), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            220 * 1024));
            PK_CUDA(h, cudaFuncSetAttribute(batched_variant<PH, FAST>(v), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            220 * 1024));
        }
        PK_CUDA(h, cudaFuncSetAttribute(fused_variant<PH, FAST>(0, true), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        220 * 1024));
        PK_CUDA(h, cudaFuncSetAttribute(batched_variant<PH, FAST>(0, true),
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024));
        PK_CUDA(h, cudaFuncSetAttribute(k_sweep_staged<PH, FAST>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        220 * 1024));
        done = true;
    }
    return PK_OK;
}

// the batched stage kernel of launch-bound variant v (SV_T / SV_B); WENO3
// runs variant 0 only
template <class PH>
auto stage_batched_variant(int v, bool w3, bool fc) -> decltype(&k_stage_batched<PH, 320, 1, false, false>)
{
    if (w3) return fc ? k_stage_batched<PH, 320, 1, true, true> : k_stage_batched<PH, 320, 1, true, false>;
    switch (v) {
    case 1: return fc ? k_stage_batched<PH, 128, 3, false, true> : k_stage_batched<PH, 128, 3, false, false>;
    case 2: return fc ? k_stage_batched<PH, 192, 2, false, true> : k_stage_batched<PH, 192, 2, false, false>;
    case 3: return fc ? k_stage_batched<PH, 384, 1, false, true> : k_stage_batched<PH, 384, 1, false, false>;
    default: return fc ? k_stage_batched<PH, 320, 1, false, true> : k_stage_batched<PH, 320, 1, false, false>;
    }
}

// the one-launch refined stage kernel of launch-bound variant v (SV_T / SV_B)
template <class PH>
auto stage_refined_variant(int v, bool w3) -> decltype(&k_stage_refined<PH, 320, 1, false>)
{
    if (w3) return k_stage_refined<PH, 320, 1, true>;
    switch (v) {
    case 1: return k_stage_refined<PH, 128, 3, false>;
    case 2: return k_stage_refined<PH, 192, 2, false>;
    case 3: return k_stage_refined<PH, 384, 1, false>;
    default: return k_stage_refined<PH, 320, 1, false>;
    }
}

template <class PH>
int set_smem_attr(pk_ctx* h)
{
    static bool done = false;
    if (!done) {
        if (int rc = set_fused_attr<PH, false>(h)) return rc;
        PK_CUDA(h, cudaFuncSetAttribute(k_stage<PH, STAGE_MAXT>, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024));
        PK_CUDA(h, cudaFuncSetAttribute(k_stage<PH, STAGE_MAXT, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        220 * 1024));
        PK_CUDA(h, cudaFuncSetAttribute(k_stage<PH, STAGE_MAXT, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        220 * 1024));
        PK_CUDA(h, cudaFuncSetAttribute(k_stage<PH, STAGE_MAXT, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        220 * 1024));
        for (auto* kf : {k_unsplit_flux<PH, UNSPLIT_MAXT, false, false>, k_unsplit_flux<PH, UNSPLIT_MAXT, true, false>,
                         k_unsplit_flux<PH, UNSPLIT_MAXT, false, true>, k_unsplit_flux<PH, UNSPLIT_MAXT, true, true>})
            PK_CUDA(h, cudaFuncSetAttribute(kf, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024));
        for (int v = 0; v < NSTAGE_VARIANT; ++v)
            for (int w3 = 0; w3 < 2; ++w3)
                for (int fc = 0; fc < 2; ++fc)
                    PK_CUDA(h, cudaFuncSetAttribute(stage_batched_variant<PH>(v, w3, fc),
                                                    cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024));
        for (int v = 0; v < NSTAGE_VARIANT; ++v)
            for (int w3 = 0; w3 < 2; ++w3)
                PK_CUDA(h, cudaFuncSetAttribute(stage_refined_variant<PH>(v, w3),
                                                cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024));
        done = true;
    }
    return PK_OK;
}

constexpr int DEF_VARIANT[3] = {0, 0, 0};
constexpr int DEF_P[3] = {2, 4, 4};
constexpr int DEF_L[3] = {64, 64, 64};

// Tile, grid and variant of the fused sweep along dir (the handle's tuned or
// default settings; a whole periodic pencil runs without halo when it fits).
// VAR_STAGED: the TMA-staged kernel where it can run (staged != 0 and
// staged_ok), otherwise the whole-pencil tile of the 256 x 2 variant.
inline int fused_geometry(pk_ctx* h, const Block& b, int dir, const Geom& g, Tile* tl, dim3* grid, int* var_out,
                          bool staged = false)
{
    int L = h->tileL[dir] > 0 ? h->tileL[dir] : DEF_L[dir];
    if (L > b.n[dir]) L = b.n[dir];
    int P = h->tileP[dir] > 0 ? h->tileP[dir] : DEF_P[dir];
    if (P > g.n1) P = g.n1;
    int var = h->pp.weno3 ? W3_VARIANT : (h->tileV[dir] >= 0 ? h->tileV[dir] : DEF_VARIANT[dir]);
    tl->wrap = h->connected ? 0 : 1;
    if (var == VAR_STAGED) {
        if (staged && tl->wrap && staged_ok(b.n, b.g, b.ext, h->nplanes, dir, g.seg_len)) {
            tl->P = 2;
            tl->T = b.n[dir];
            tl->L = b.n[dir];
            tl->circ = 1;
            tl->halo = 0;
            tl->xfast = (dir == 0);
            *grid = dim3((g.n1 + 1) / 2, 1, g.n2);
            *var_out = VAR_STAGED;
            return PK_OK;
        }
        var = 2;
        L = b.n[dir] <= VAR_T[2] ? b.n[dir] : VAR_T[2] - 8;
        P = 1;
    }
    const int maxt = VAR_T[var];
    tl->circ = (tl->wrap && L == b.n[dir] && b.n[dir] <= maxt) ? 1 : 0;
    if (g.seg_len && g.seg_along) {                   // stacked instances: one whole segment per tile
        L = g.seg_len;
        tl->circ = 1;
        if (L > maxt) return fail(h, PK_E_ARG, "instance segment longer than the variant's CTA size");
    }
    const int T = tl->circ ? L : L + 8;
    while (P * T > maxt && P > 1) --P;
    if (P * T > maxt) return fail(h, PK_E_ARG, "fused sweep tile longer than the variant's CTA size");
    tl->P = P;
    tl->T = T;
    tl->L = L;
    tl->halo = 4;
    tl->xfast = (dir == 0);
    *grid = dim3((g.n1 + P - 1) / P, (b.n[dir] + L - 1) / L, g.n2);
    *var_out = var;
    return PK_OK;
}

template <class PH, bool FAST = false>
int launch_fused_ptr(pk_ctx* h, Block& b, int dir, int apply_fac, const double* in, double* out)
{
    if (int rc = set_fused_attr<PH, FAST>(h)) return rc;
    Geom g = make_geom(b, dir);
    Tile tl;
    dim3 grid;
    int var;
    if (int rc = fused_geometry(h, b, dir, g, &tl, &grid, &var, !h->pp.weno3)) return rc;
    std::pair<cudaEvent_t, cudaEvent_t> ev;
    if (var == VAR_STAGED) {
        CUtensorMap tin, tout;
        if (!encode_state_map(&tin, in, b.n, b.ext, b.plane, PH::NV, dir) ||
            !encode_state_map(&tout, out, b.n, b.ext, b.plane, PH::NV, dir))
            return fail(h, PK_E_CUDA, "cuTensorMapEncodeTiled failed for the staged sweep");
        const int threads = (b.n[dir] + 31) / 32 * 32;
        if (int rc = ev_begin(h, &ev)) return fail(h, rc, "cudaEventRecord failed");
        k_sweep_staged<PH, FAST><<<grid, threads, staged_smem(PH::NV, b.n[dir]), h->stream>>>(
            tin, tout, g, h->pp, b.dl[dir], h->d_step, apply_fac, dir, h->d_status, nullptr, nullptr);
    } else {
        const size_t smem = 3ull * PH::NV * tl.P * tl.T * sizeof(double);
        if (int rc = ev_begin(h, &ev)) return fail(h, rc, "cudaEventRecord failed");
        fused_variant<PH, FAST>(var, h->pp.weno3)<<<grid, tl.P * tl.T, smem, h->stream>>>(g, tl, in, out, h->pp,
                                                                                         b.dl[dir], h->d_step,
                                                                                         apply_fac, h->d_status);
    }
    PK_CUDA(h, cudaGetLastError());
    if (int rc = ev_end(h, ev)) return fail(h, rc, "cudaEventRecord failed");
    h->launches += 1;
    return PK_OK;
}

template <class PH, bool FAST = false>
int launch_fused(pk_ctx* h, Block& b, int dir, int apply_fac)
{
    if (int rc = launch_fused_ptr<PH, FAST>(h, b, dir, apply_fac, b.buf[h->cur], b.buf[1 - h->cur])) return rc;
    b.guards_stale = true;
    return PK_OK;
}

template <class PH>
using RecFn = void (*)(Geom, Tile, const double*, double*, double*, unsigned short*, PhysParams, double,
                       const StepParams*, int, unsigned*);

template <class PH>
RecFn<PH> rec_variant(int v)
{
    switch (v) {
    case 0: return k_sweep_fused_rec<PH, 320, 1>;
    case 1: return k_sweep_fused_rec<PH, 256, 1>;
    case 2: return k_sweep_fused_rec<PH, 256, 2>;
    case 3: return k_sweep_fused_rec<PH, 128, 3>;
    case 4: return k_sweep_fused_rec<PH, 128, 4>;
    case 5: return k_sweep_fused_rec<PH, 192, 2>;
    case 6: return k_sweep_fused_rec<PH, 512, 1>;
    default: return k_sweep_fused_rec<PH, 256, 2>;
    }
}

// The forward sweep of the backward pass's recomputation, in the forward
// sweep's tile and variant (the TMA-staged kernel where the forward's tile is
// the staged one): also stores U* and the floor records
template <class PH>
int launch_fused_rec(pk_ctx* h, Block& b, int dir, int apply_fac, const double* in, double* out, double* ustar,
                     unsigned short* flags)
{
    if constexpr (PH::NFL != 1) {
        return fail(h, PK_E_UNSUPPORTED, "the differentiable path is built for one-fluid HD and MHD");
    } else {
        static bool attr = false;
        if (!attr) {
            for (int v = 0; v < NVARIANT; ++v)
                PK_CUDA(h, cudaFuncSetAttribute(rec_variant<PH>(v), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                220 * 1024));
            PK_CUDA(h, cudaFuncSetAttribute(k_sweep_staged<PH, false, true>,
                                            cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024));
            attr = true;
        }
        Geom g = make_geom(b, dir);
        Tile tl;
        dim3 grid;
        int var;
        if (int rc = fused_geometry(h, b, dir, g, &tl, &grid, &var, true)) return rc;
        std::pair<cudaEvent_t, cudaEvent_t> ev;
        if (var == VAR_STAGED) {
            CUtensorMap tin, tout;
            if (!encode_state_map(&tin, in, b.n, b.ext, b.plane, PH::NV, dir) ||
                !encode_state_map(&tout, out, b.n, b.ext, b.plane, PH::NV, dir))
                return fail(h, PK_E_CUDA, "cuTensorMapEncodeTiled failed for the staged sweep");
            const int threads = (b.n[dir] + 31) / 32 * 32;
            if (int rc = ev_begin(h, &ev)) return fail(h, rc, "cudaEventRecord failed");
            k_sweep_staged<PH, false, true><<<grid, threads, staged_smem(PH::NV, b.n[dir]), h->stream>>>(
                tin, tout, g, h->pp, b.dl[dir], h->d_step, apply_fac, dir, h->d_status, ustar, flags);
        } else {
            const size_t smem = 3ull * PH::NV * tl.P * tl.T * sizeof(double);
            if (int rc = ev_begin(h, &ev)) return fail(h, rc, "cudaEventRecord failed");
            rec_variant<PH>(var)<<<grid, tl.P * tl.T, smem, h->stream>>>(g, tl, in, out, ustar, flags, h->pp,
                                                                        b.dl[dir], h->d_step, apply_fac, h->d_status);
        }
        PK_CUDA(h, cudaGetLastError());
        if (int rc = ev_end(h, ev)) return fail(h, rc, "cudaEventRecord failed");
        h->launches += 1;
        return PK_OK;
    }
}

// Launch-bound variants of the two adjoint kernels (threads per CTA, CTAs per
// SM); variant ADJ_VAR_STAGED is the TMA-staged whole-pencil pair
// (k_adj_staged2 / k_adj_staged1: two pencils per CTA, n <= 256 and the
// staged forward kernel's alignment conditions; elsewhere variant 0)
constexpr int NADJ_VARIANT = 6;
constexpr int ADJ_VAR_STAGED = 5;
constexpr int ADJ_T[NADJ_VARIANT] = {256, 256, 192, 128, 128, 256};
// defaults, measured on B200 (MHD, 256^3, adjoint sweep = staged recording
// sweep + the two adjoint kernels): the staged pair 10.9 / 12.5 / 13.0 ms
// along x / y / z against 12.5 / 15.8 / 16.2 for the best tiled variant
// (persistent double-buffered stage 2 everywhere; stage 1 persistent along x,
// one tile per CTA with lam staged along y and z: the persistent stage 1's
// plain lam accesses there cost 14.5 / 14.8 ms).
// Among the tiled variants (where the staged pair does not apply) the
// unspilled 255-register variant 0 is the fastest or within 1 % of it on
// every axis; the whole periodic pencil without halo beats 8 pencils x 26 + 6
// halo cells along x and along y and z while at least two pencils share the
// CTA, but not with one pencil per CTA (250-cell chunks along y: 33.5 ms
// against 19.0), and chunks that do not divide the pencil waste their last
// tile (58 cells: 19.4 ms along y)
constexpr int DEF_ADJ_V[3] = {ADJ_VAR_STAGED, ADJ_VAR_STAGED, ADJ_VAR_STAGED};
constexpr int DEF_ADJ_CHUNK = 26;

inline int default_adj_length(int dir, int n, int threads)
{
    if (n <= threads && (dir == 0 || 2 * n <= threads)) return n;
    return DEF_ADJ_CHUNK;
}

template <class PH>
struct AdjKernels {
    decltype(&k_adj_stage2<PH, 256, 1>) s2;
    decltype(&k_adj_stage1<PH, 256, 1>) s1;
};

template <class PH>
AdjKernels<PH> adj_variant(int v)
{
    switch (v) {
    case 0: return {k_adj_stage2<PH, 256, 1>, k_adj_stage1<PH, 256, 1>};
    case 1: return {k_adj_stage2<PH, 256, 2>, k_adj_stage1<PH, 256, 2>};
    case 2: return {k_adj_stage2<PH, 192, 2>, k_adj_stage1<PH, 192, 2>};
    case 3: return {k_adj_stage2<PH, 128, 3>, k_adj_stage1<PH, 128, 3>};
    default: return {k_adj_stage2<PH, 128, 4>, k_adj_stage1<PH, 128, 4>};
    }
}

// Adjoint of one fused sweep: lam_in = (d sweep / d uin)^T lam_out, from the
// sweep's input, its stage-1 state, its output and floor records; m1 is
// scratch of one state.
template <class PH>
int launch_adj(pk_ctx* h, Block& b, int dir, int apply_fac, const double* uin, const double* ustar, const double* uout,
               const unsigned short* flags, const double* lam_out, double* lam_in, double* m1)
{
    if constexpr (PH::NFL != 1) {
        return fail(h, PK_E_UNSUPPORTED, "the adjoint sweep is built for one-fluid HD and MHD");
    } else {
        static bool attr = false;
        if (!attr) {
            for (int v = 0; v < ADJ_VAR_STAGED; ++v) {
                const AdjKernels<PH> k = adj_variant<PH>(v);
                PK_CUDA(h, cudaFuncSetAttribute(k.s2, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024));
                PK_CUDA(h, cudaFuncSetAttribute(k.s1, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024));
            }
            PK_CUDA(h, cudaFuncSetAttribute(k_adj_staged2<PH>, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024));
            PK_CUDA(h, cudaFuncSetAttribute(k_adj_staged1<PH>, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024));
            PK_CUDA(h, cudaFuncSetAttribute(k_adj_staged1_boxed<PH>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            220 * 1024));
            attr = true;
        }
        int var = (h->adjV[dir] >= 0 && h->adjV[dir] < NADJ_VARIANT) ? h->adjV[dir] : DEF_ADJ_V[dir];
        Geom g = make_geom(b, dir);
        if (var == ADJ_VAR_STAGED) {
            if (staged_ok(b.n, b.g, b.ext, h->nplanes, dir, g.seg_len)) {
                CUtensorMap m_ustar, m_lamout, m_lamin, m_m1, m_uin;
                if (!encode_state_map(&m_ustar, ustar, b.n, b.ext, b.plane, PH::NV, dir) ||
                    !encode_state_map(&m_lamout, lam_out, b.n, b.ext, b.plane, PH::NV, dir) ||
                    !encode_state_map(&m_lamin, lam_in, b.n, b.ext, b.plane, PH::NV, dir) ||
                    !encode_state_map(&m_m1, m1, b.n, b.ext, b.plane, PH::NV, dir) ||
                    !encode_state_map(&m_uin, uin, b.n, b.ext, b.plane, PH::NV, dir))
                    return fail(h, PK_E_CUDA, "cuTensorMapEncodeTiled failed for the staged adjoint sweep");
                const int threads = (b.n[dir] + 31) / 32 * 32;
                // persistent: as many CTAs as can be resident (one per SM at
                // 256 threads, more for shorter pencils), over the tiles (pairs of pencils)
                const long long ntiles = (long long)((g.n1 + 1) / 2) * g.n2;
                const size_t smem = adj_staged_smem(PH::NV, b.n[dir]);
                int per_sm = 0;
                PK_CUDA(h, cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                               &per_sm, dir == 0 ? (const void*)k_adj_staged1<PH> : (const void*)k_adj_staged2<PH>,
                               threads, smem));
                if (per_sm < 1) per_sm = 1;
                const int ctas = (int)std::min<long long>(ntiles, (long long)per_sm * sm_count());
                std::pair<cudaEvent_t, cudaEvent_t> ev;
                if (int rc = ev_begin(h, &ev)) return fail(h, rc, "cudaEventRecord failed");
                k_adj_staged2<PH><<<ctas, threads, smem, h->stream>>>(m_ustar, m_lamout, m_lamin, m_m1, g, uout,
                                                                      flags, h->pp, b.dl[dir], h->d_step,
                                                                      apply_fac, dir, h->d_status);
                PK_CUDA(h, cudaGetLastError());
                if (dir == 0) {
                    k_adj_staged1<PH><<<ctas, threads, smem, h->stream>>>(m_uin, m_m1, g, lam_in, h->pp, h->d_step,
                                                                          dir, h->d_status);
                } else {
                    const dim3 grid((g.n1 + 1) / 2, 1, g.n2);
                    k_adj_staged1_boxed<PH><<<grid, threads, adj_staged1_boxed_smem(PH::NV, b.n[dir]), h->stream>>>(
                        m_uin, m_m1, m_lamin, g, h->pp, h->d_step, dir, h->d_status);
                }
                PK_CUDA(h, cudaGetLastError());
                if (int rc = ev_end(h, ev)) return fail(h, rc, "cudaEventRecord failed");
                h->launches += 2;
                return PK_OK;
            }
            var = 0;                                  // not stageable here: the tiled default
        }
        Tile tl;
        int L = h->adjL[dir] > 0 ? h->adjL[dir] : default_adj_length(dir, b.n[dir], ADJ_T[var]);
        if (L > b.n[dir]) L = b.n[dir];
        tl.circ = (L == b.n[dir] && b.n[dir] <= ADJ_T[var]) ? 1 : 0;
        if (g.seg_len && g.seg_along) {               // stacked instances: one whole segment per tile
            L = g.seg_len;
            tl.circ = 1;
            if (L > ADJ_T[var]) return fail(h, PK_E_ARG, "instance segment longer than the adjoint variant's CTA size");
        }
        if (!tl.circ && L > ADJ_T[var] - 6) L = ADJ_T[var] - 6;
        tl.T = tl.circ ? L : L + 6;
        tl.P = ADJ_T[var] / tl.T;
        if (tl.P < 1) return fail(h, PK_E_ARG, "adjoint tile longer than the variant's CTA size");
        if (tl.P > g.n1) tl.P = g.n1;
        tl.L = L;
        tl.halo = 3;
        tl.xfast = dir == 0;
        dim3 grid((g.n1 + tl.P - 1) / tl.P, (b.n[dir] + tl.L - 1) / tl.L, g.n2);
        const size_t smem = 4ull * PH::NV * tl.P * tl.T * sizeof(double);
        const AdjKernels<PH> k = adj_variant<PH>(var);
        std::pair<cudaEvent_t, cudaEvent_t> ev;
        if (int rc = ev_begin(h, &ev)) return fail(h, rc, "cudaEventRecord failed");
        k.s2<<<grid, tl.P * tl.T, smem, h->stream>>>(g, tl, ustar, uout, flags, lam_out, lam_in, m1, h->pp, b.dl[dir],
                                                     h->d_step, apply_fac);
        PK_CUDA(h, cudaGetLastError());
        k.s1<<<grid, tl.P * tl.T, smem, h->stream>>>(g, tl, uin, m1, lam_in, h->pp, h->d_step);
        PK_CUDA(h, cudaGetLastError());
        if (int rc = ev_end(h, ev)) return fail(h, rc, "cudaEventRecord failed");
        h->launches += 2;
        return PK_OK;
    }
}

template <class PH, bool FAST = false>
int launch_batched(pk_ctx* h, int dir, int apply_fac, unsigned* counter)
{
    if (int rc = set_fused_attr<PH, FAST>(h)) return rc;
    BatchList& bl = h->batch[dir];
    if (bl.n == 0) return PK_OK;
    const int var = h->pp.weno3 ? W3_VARIANT : h->batch_variant;
    int maxP = 1;
    for (const auto& w : bl.host) maxP = (w.P * (w.L + 8) > maxP) ? w.P * (w.L + 8) : maxP;
    const int threads = VAR_T[var];
    const size_t smem = 3ull * PH::NV * threads * sizeof(double);
    int dev = 0, nsm = 0, per_sm = 0;
    PK_CUDA(h, cudaGetDevice(&dev));
    PK_CUDA(h, cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    PK_CUDA(h, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batched_variant<PH, FAST>(var, h->pp.weno3),
                                                             threads, smem));
    if (per_sm < 1) return fail(h, PK_E_ARG, "batched sweep tile does not fit on an SM");
    int grid = nsm * per_sm;
    if (grid > bl.n) grid = bl.n;
    PK_CUDA(h, cudaMemsetAsync(counter, 0, sizeof(unsigned), h->stream));
    std::pair<cudaEvent_t, cudaEvent_t> ev;
    if (int rc = ev_begin(h, &ev)) return fail(h, rc, "cudaEventRecord failed");
    batched_variant<PH, FAST>(var, h->pp.weno3)<<<grid, threads, smem, h->stream>>>(
        h->d_desc[h->cur], bl.dev, bl.n, dir, h->pp, h->d_step, apply_fac, counter, h->d_status);
    PK_CUDA(h, cudaGetLastError());
    if (int rc = ev_end(h, ev)) return fail(h, rc, "cudaEventRecord failed");
    h->launches += 1;
    (void)maxP;
    return PK_OK;
}

template <class PH>
int launch_stage(pk_ctx* h, Block& b, int dir, int first, double rk)
{
    if (int rc = set_smem_attr<PH>(h)) return rc;
    Geom g = make_geom(b, dir);
    Tile tl;
    const int ext = b.ext[dir];
    double* u = b.buf[h->cur];
    double* uout = u;
    if (!stage_chunked(b, dir)) {            // whole pencils per tile: in place
        int P = STAGE_MAXT / ext;
        if (P >= 4) P -= P % 4;
        if (P > g.n1) P = g.n1;
        tl.P = P;
        tl.T = ext;
        tl.L = ext;
        tl.halo = 0;
    } else {                                 // chunked with a 2-cell halo: out of place
        tl.P = 4;
        tl.L = 64;
        tl.T = tl.L + 4;
        tl.halo = 2;
        uout = b.buf[1 - h->cur];
    }
    tl.xfast = (dir == 0);
    dim3 grid((g.n1 + tl.P - 1) / tl.P, (ext + tl.L - 1) / tl.L, g.n2);
    const size_t smem = 3ull * PH::NV * tl.P * tl.T * sizeof(double);
    std::pair<cudaEvent_t, cudaEvent_t> ev;
    if (int rc = ev_begin(h, &ev)) return fail(h, rc, "cudaEventRecord failed");
    const FcArgs& fc = b.fc[dir];
    const bool hooks = fc.in_slot || fc.out_slot;      // a fine/coarse boundary crosses this block's pencils
    auto* kern = h->pp.weno3 ? (hooks ? k_stage<PH, STAGE_MAXT, true, true> : k_stage<PH, STAGE_MAXT, true, false>)
                             : (hooks ? k_stage<PH, STAGE_MAXT, false, true> : k_stage<PH, STAGE_MAXT, false, false>);
    kern<<<grid, tl.P * tl.T, smem, h->stream>>>(g, tl, u, uout, b.uh, h->pp, first, rk, b.dl[dir], h->d_step,
                                                 h->d_status, fc);
    PK_CUDA(h, cudaGetLastError());
    if (int rc = ev_end(h, ev)) return fail(h, rc, "cudaEventRecord failed");
    h->launches += 1;
    if (uout != u) {
        BoxGeom bg;
        for (int d = 0; d < 3; ++d) {
            bg.ext[d] = b.ext[d];
            bg.g[d] = b.g[d];
            bg.n[d] = b.n[d];
        }
        bg.plane = b.plane;
        long long nb = (b.plane + 255) / 256;
        if (nb > grid_cap()) nb = grid_cap();
        k_copy_pencils<<<(int)nb, 256, 0, h->stream>>>(bg, dir, uout, u, h->nplanes);
        PK_CUDA(h, cudaGetLastError());
        h->launches += 1;
    }
    return PK_OK;
}

// one stage of every block of a level in one launch (k_stage_batched); the
// work list and the block table were built by build_batch
template <class PH>
int launch_stage_batched(pk_ctx* h, int dir, int level, int first, double rk)
{
    if (level >= (int)h->sbatch[dir].size()) return PK_OK;
    const StageList& sl = h->sbatch[dir][level];
    if (!sl.n) return PK_OK;
    if (int rc = set_smem_attr<PH>(h)) return rc;
    const bool hooks = h->d_fcargs[dir] != nullptr;
    const int v = h->pp.weno3 ? 0 : h->stage_variant;
    auto* kern = stage_batched_variant<PH>(v, h->pp.weno3, hooks);
    std::pair<cudaEvent_t, cudaEvent_t> ev;
    if (int rc = ev_begin(h, &ev)) return fail(h, rc, "cudaEventRecord failed");
    kern<<<sl.n, SV_T[v], sl.smem, h->stream>>>(h->d_desc[h->cur], sl.dev, dir, h->pp, first, rk, h->d_step,
                                               h->d_fcargs[dir], h->d_status);
    PK_CUDA(h, cudaGetLastError());
    if (int rc = ev_end(h, ev)) return fail(h, rc, "cudaEventRecord failed");
    h->launches += 1;
    return PK_OK;
}

// One stage of every level of a refined domain along dir in one persistent
// launch (k_stage_refined): as many CTAs as can be resident, at most one per
// work item; its counters are zeroed on the stream first.
template <class PH>
int launch_stage_refined(pk_ctx* h, int dir, int first, double rk)
{
    const int n = h->rn[dir];
    if (!n) return PK_OK;
    if (int rc = set_smem_attr<PH>(h)) return rc;
    const int v = h->pp.weno3 ? 0 : h->stage_variant;
    auto* kern = stage_refined_variant<PH>(v, h->pp.weno3);
    const size_t smem = h->rsmem[dir];
    int per_sm = 0;
    PK_CUDA(h, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, SV_T[v], smem));
    if (per_sm < 1) return fail(h, PK_E_CUDA, "the refined stage kernel does not fit an SM");
    const int ctas = std::min(n, per_sm * sm_count());
    RefArgs ra;
    ra.src = h->d_src[dir];
    ra.out_flux = h->d_out_flux[dir];
    ra.in_flux = h->d_in_flux[dir];
    ra.scale = h->fc_scale;
    ra.nlev = h->max_level + 1;
    PK_CUDA(h, cudaMemsetAsync(h->d_rcount, 0, sizeof(unsigned) * h->rcount_n, h->stream));
    std::pair<cudaEvent_t, cudaEvent_t> ev;
    if (int rc = ev_begin(h, &ev)) return fail(h, rc, "cudaEventRecord failed");
    kern<<<ctas, SV_T[v], smem, h->stream>>>(h->d_desc[h->cur], h->rdev[dir], n, dir, h->pp, first, rk, h->d_step,
                                             h->d_fcargs[dir], ra, h->d_rcount, h->d_status);
    PK_CUDA(h, cudaGetLastError());
    if (int rc = ev_end(h, ev)) return fail(h, rc, "cudaEventRecord failed");
    h->launches += 1;
    return PK_OK;
}

// the face fluxes of one direction for the unsplit scheme (k_unsplit_flux),
// tiles as the stage kernel's
template <class PH>
int launch_unsplit_flux(pk_ctx* h, Block& b, int dir, const double* in, double* F)
{
    if (int rc = set_smem_attr<PH>(h)) return rc;
    Geom g = make_geom(b, dir);
    Tile tl;
    const int ext = b.ext[dir];
    // whole pencils where they fit; across x (y and z sweeps) only when four or
    // more neighbouring pencils share the CTA, so that the loads stay coalesced,
    // else chunks of 64 cells with a 2-cell halo
    if (ext <= UNSPLIT_MAXT && (dir == 0 || UNSPLIT_MAXT / ext >= 4 || g.n1 < 4)) {
        int P = UNSPLIT_MAXT / ext;
        if (P >= 4) P -= P % 4;
        if (P > g.n1) P = g.n1;
        tl.P = P;
        tl.T = ext;
        tl.L = ext;
        tl.halo = 0;
    } else {
        tl.P = 4;
        tl.L = UNSPLIT_MAXT / 4 - 4;
        tl.T = tl.L + 4;
        tl.halo = 2;
    }
    tl.xfast = (dir == 0);
    dim3 grid((g.n1 + tl.P - 1) / tl.P, (ext + tl.L - 1) / tl.L, g.n2);
    const size_t smem = 3ull * PH::NV * tl.P * tl.T * sizeof(double);
    std::pair<cudaEvent_t, cudaEvent_t> ev;
    if (int rc = ev_begin(h, &ev)) return fail(h, rc, "cudaEventRecord failed");
    // a refined block's fine/coarse flux couplings along dir (ext_fluxes, unsplit_mag_modules.F90:195-204)
    const FcArgs fc = b.fc[dir];
    const bool hooks = fc.in_slot || fc.out_slot;
    auto* kern = h->pp.weno3 ? (hooks ? k_unsplit_flux<PH, UNSPLIT_MAXT, true, true> : k_unsplit_flux<PH, UNSPLIT_MAXT, true, false>)
                             : (hooks ? k_unsplit_flux<PH, UNSPLIT_MAXT, false, true> : k_unsplit_flux<PH, UNSPLIT_MAXT, false, false>);
    kern<<<grid, tl.P * tl.T, smem, h->stream>>>(g, tl, in, F, h->pp, h->d_step, h->d_status, fc);
    PK_CUDA(h, cudaGetLastError());
    if (int rc = ev_end(h, ev)) return fail(h, rc, "cudaEventRecord failed");
    h->launches += 1;
    return PK_OK;
}

template <class PH>
int launch_unsplit_apply(pk_ctx* h, Block& b, const double* S, double* T, double rk, int last)
{
    BoxGeom bg;
    for (int d = 0; d < 3; ++d) {
        bg.ext[d] = b.ext[d];
        bg.g[d] = b.g[d];
        bg.n[d] = b.n[d];
    }
    bg.plane = b.plane;
    long long nblk = (b.plane + 255) / 256;
    if (nblk > grid_cap()) nblk = grid_cap();
    k_unsplit_apply<PH><<<(int)nblk, 256, 0, h->stream>>>(bg, S, T, b.flux[0], b.flux[1], b.flux[2], h->pp, h->d_step,
                                                          rk, b.dl[0], b.dl[1], b.dl[2], last, h->d_status);
    PK_CUDA(h, cudaGetLastError());
    h->launches += 1;
    return PK_OK;
}

// the tolerance-mode sweeps of PH (instantiated by the pk_fast_*.cu units only)
template <class PH>
const FastOps* make_fast_ops()
{
    static FastOps o{set_fused_attr<PH, true>, launch_fused<PH, true>, launch_batched<PH, true>};
    return &o;
}

template <class PH>
const PhysOps* make_ops()
{
    static PhysOps o{PH::NV, set_smem_attr<PH>, launch_fused<PH>, launch_stage<PH>, launch_stage_batched<PH>,
                     launch_stage_refined<PH>, launch_batched<PH>, launch_fused_ptr<PH>, launch_fused_rec<PH>, launch_adj<PH>,
                     launch_unsplit_flux<PH>, launch_unsplit_apply<PH>};
    return &o;
}

}  // namespace pk
