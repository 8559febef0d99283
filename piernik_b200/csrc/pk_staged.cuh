// pk_staged.cuh -- the fused two-stage sweep of a periodic block over whole
// pencils staged in shared memory by the tensor memory accelerator (TMA).
//
// A CTA owns two neighbouring pencils (ortho-1 indices i1_0, i1_0 + 1 at
// ortho-2 index i2), whole along the sweep direction (n <= 256 cells).  One
// thread issues a single cp.async.bulk.tensor load of the box
// [2 pencils x n cells x all component planes] from a 4-D tensor map of the
// block (x, y, z, plane); for y and z sweeps each of its rows is 16 contiguous
// bytes that the TMA engine gathers asynchronously, so no warp issues a
// strided load.  The CTA then sweeps the two pencils one after the other
// (pass 0, pass 1) with the circular whole-pencil tile of the fused kernel
// (no halo, nothing computed twice): the cell's state comes from the staged
// box, the RK2 update reads u0 from it too, and the result goes back into the
// box over the cell's own input.  A cp.async.bulk.tensor store then writes the
// box to the output state.  The arithmetic per cell is fused_tile's
// (pk_kernels.cuh) exactly, so results equal the other fused kernels bit for
// bit (or, in the tolerance mode, the other tolerance-mode kernels).
//
// Requirements (checked on the host before the launch): a single periodic
// block read with wrap (not connected; stacked instances only along x and y,
// each CTA taking its instance's step scalars), n <= 256 along
// the sweep, an even x extent and an even x guard width (the box's x
// coordinate and the tensor strides must be multiples of 16 bytes), linear
// reconstruction.  Shared memory: 2n planes-worth of doubles for the box plus
// the three n-cell planes of the tile per component.
//
// REC (the backward pass's recomputation, bit-exact arithmetic only): also
// store each cell's stage-1 state in ustar and its floor records in flags, as
// k_sweep_fused_rec does; these go out with plain stores at the cell's own
// offset.
//
// The wait for the load is bounded: a CTA that gives up raises
// PK_ST_TIMEOUT in the status word and returns without touching the output.
#pragma once
#include <cuda.h>

#include "pk_kernels.cuh"

namespace pk {

constexpr unsigned ST_TIMEOUT = 4u;   // PK_ST_TIMEOUT

PK_DEV unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

PK_DEV void mbar_init(unsigned long long* bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

PK_DEV void mbar_expect_tx(unsigned long long* bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// true once the barrier's phase `parity` has completed
PK_DEV bool mbar_try_wait(unsigned long long* bar, unsigned parity)
{
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

PK_DEV void tma_load_4d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, int c3, unsigned long long* bar)
{
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
        "[%6];" ::"r"(smem_u32(dst)),
        "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
        : "memory");
}

PK_DEV void tma_store_4d(const CUtensorMap* map, const void* src, int c0, int c1, int c2, int c3)
{
    asm volatile("cp.async.bulk.tensor.4d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3, %4}], [%5];" ::"l"(map),
                 "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(src))
                 : "memory");
    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}

// this thread's shared-memory writes become visible to the TMA engine
PK_DEV void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// ---------------------------------------------------------------------------
// grid: x = pairs of pencils along ortho-1, y = 1, z = ortho-2; blockDim.x >= n
// ---------------------------------------------------------------------------
template <class PH, bool FAST = false, bool REC = false>
__global__ void __launch_bounds__(256, 2) k_sweep_staged(const __grid_constant__ CUtensorMap tin,
                                                         const __grid_constant__ CUtensorMap tout, Geom g,
                                                         PhysParams pp, double dl, const StepParams* __restrict__ sp,
                                                         int apply_fac, int dir, unsigned* __restrict__ gstatus,
                                                         double* __restrict__ ustar, unsigned short* __restrict__ flags)
{
    static_assert(!(REC && FAST), "the recording sweep runs in the bit-exact arithmetic");
    constexpr int NV = PH::NV;
    extern __shared__ __align__(128) double smem[];
    const int n = g.n_d;
    double* box = smem;                                  // [NV][2n] in the box's element order
    const Smem sm{box + 2 * NV * n, box + 3 * NV * n, box + 4 * NV * n, n};
    unsigned long long* bar = reinterpret_cast<unsigned long long*>(box + 5 * NV * n);
    // element strides of the box along the pencil (t) and across the pair (p)
    const int st_t = dir == 0 ? 1 : 2, st_p = dir == 0 ? n : 1;
    const int i1_0 = 2 * blockIdx.x, i2 = blockIdx.z;
    const int o1 = dir == 0 ? 1 : 0, o2 = dir == 2 ? 1 : 2;
    int c[4];
    c[dir] = g.g_d;
    c[o1] = g.g1 + i1_0;
    c[o2] = g.g2 + i2;
    c[3] = 0;
    const int tid = threadIdx.x;
    if (tid == 0) {
        mbar_init(bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        fence_proxy_async();
    }
    __syncthreads();
    if (tid == 0) {
        mbar_expect_tx(bar, (unsigned)(2 * NV * n * sizeof(double)));
        tma_load_4d(box, &tin, c[0], c[1], c[2], c[3], bar);
    }
    bool ready = false;
    for (int it = 0; it < (1 << 24) && !ready; ++it) ready = mbar_try_wait(bar, 0);
    if (!__syncthreads_and(ready)) {
        if (tid == 0) atomicOr(gstatus, ST_TIMEOUT);
        return;
    }

    const StepParams stp = sp[g.seg_len ? i2 / g.seg_len : 0];   // stacked instances: this CTA's
    const double dtodx1 = (0.5 * stp.dt) / dl;           // rk_coef(RK2_1) * dt / cg%dl(ddim)
    const double dtodx2 = (1.0 * stp.dt) / dl;           // rk_coef(RK2_2) * dt / cg%dl(ddim)
    const double ch = stp.ch, psi_fac = apply_fac ? stp.psi_fac : 1.0;
    const int perm[3] = {g.perm[0], g.perm[1], g.perm[2]};
    const int t = tid;
    const int mp = t == 0 ? n - 1 : t - 1, mn = t == n - 1 ? 0 : t + 1;
    unsigned status = 0;
    // one copy of the stage code for both pencils and both RK2 stages (the
    // solver inlined four times overflows the instruction cache)
#pragma unroll 1
    for (int p = 0; p < 2; ++p) {
        if (i1_0 + p >= g.n1) break;                     // the same for the whole CTA
        const bool active = t < n;
        double* mine = box + (active ? t : 0) * st_t + p * st_p;   // this cell's plane-0 entry in the box
        double w[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) w[v] = active ? mine[plane_of<PH>(v, perm) * 2 * n] : 0.0;
        Roles r;
        r.end = 0;
        r.keep = false;
        r.q = r.slope = r.flux = r.upd = active;
        // the cell's offset in the block (REC's plain stores)
        const long long off = (long long)(g.g_d + t) * g.sd + (long long)(g.g1 + i1_0 + p) * g.s1 +
                              (long long)(g.g2 + i2) * g.s2;
        FloorRec rec1{0, 0}, rec2{0, 0};
#pragma unroll 1
        for (int s = 0; s < 2; ++s) {
            FloorRec rec{0, 0};
            rk_stage<PH, REC, false, false, FAST, true>(sm, t, mp, mn, r, w, nullptr, nullptr, 0, g,
                                                        s == 0 ? dtodx1 : dtodx2, ch, pp, status, &rec, nullptr,
                                                        nullptr, mine, 2 * n);
            if constexpr (REC) {
                if (s == 0) {
                    rec1 = rec;
                    if (active) store_cell<PH>(ustar, off, g, w);
                } else {
                    rec2 = rec;
                }
            }
        }
        if (active) {
            if (PH::MHD) w[PH::IB + 3] = w[PH::IB + 3] * psi_fac;   // glmdamping fused into the last sweep
#pragma unroll
            for (int v = 0; v < NV; ++v) mine[plane_of<PH>(v, perm) * 2 * n] = w[v];
            if constexpr (REC) flags[off] = pack_floors(rec1, rec2);
        }
    }
    fence_proxy_async();
    __syncthreads();
    if (tid == 0) {
        tma_store_4d(&tout, box, c[0], c[1], c[2], c[3]);
        asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
    }
    flush_status(status, gstatus);
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

inline EncodeTiledFn encode_tiled_fn()
{
    static EncodeTiledFn fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    }
    return fn;
}

// whether the staged kernel can sweep block b along dir (see the requirements above)
inline bool staged_ok(const int n[3], const int g[3], const int ext[3], int nplanes, int dir, int seg_len)
{
    // stacked instances (along z) are staged along x and y, where a pencil
    // stays inside one instance; along z a pencil would cross them
    if ((seg_len && dir == 2) || n[dir] > 256 || n[dir] < 2 || nplanes > 256) return false;
    if ((ext[0] & 1) || (g[0] & 1)) return false;        // 16-byte strides and x coordinates
    if (dir == 0 && (n[0] & 1)) return false;            // the box's x rows: 16-byte multiples
    return encode_tiled_fn() != nullptr;
}

// the block's state as a 4-D tensor (x, y, z, plane) with the box of one staged tile along dir
inline bool encode_state_map(CUtensorMap* m, const double* base, const int n[3], const int ext[3], long long plane,
                             int nplanes, int dir)
{
    const int o1 = dir == 0 ? 1 : 0, o2 = dir == 2 ? 1 : 2;
    cuuint64_t dims[4] = {(cuuint64_t)ext[0], (cuuint64_t)ext[1], (cuuint64_t)ext[2], (cuuint64_t)nplanes};
    cuuint64_t strides[3] = {(cuuint64_t)ext[0] * 8, (cuuint64_t)ext[0] * ext[1] * 8, (cuuint64_t)plane * 8};
    cuuint32_t box[4];
    box[dir] = (cuuint32_t)n[dir];
    box[o1] = 2;
    box[o2] = 1;
    box[3] = (cuuint32_t)nplanes;
    cuuint32_t es[4] = {1, 1, 1, 1};
    return encode_tiled_fn()(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, const_cast<double*>(base), dims, strides, box, es,
                             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                             CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// dynamic shared memory of a staged tile of nv planes and n cells (+ the mbarrier)
inline size_t staged_smem(int nv, int n) { return (size_t)5 * nv * n * sizeof(double) + 16; }

}  // namespace pk
