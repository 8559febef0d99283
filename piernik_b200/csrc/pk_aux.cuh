// pk_aux.cuh -- bandwidth kernels around the sweep: CFL reduction, psi
// damping, guard-cell refresh, host-layout conversion.
#pragma once
#include "../../include/piernik_b200.h"
#include "pk_device.cuh"
#include "pk_kernels.cuh"

namespace pk {

struct BoxGeom {
    int ext[3], g[3], n[3];
    long long plane;
};

PK_DEV long long cell_index(const BoxGeom& b, int i, int j, int k)
{
    return ((long long)k * b.ext[1] + j) * b.ext[0] + i;
}

struct CflFluid {
    int kind;        // K_ION / K_NEU / K_DST
    int beg;         // first component plane of the fluid
    double gam, gam_1;
};

struct CflArgs {
    int nfl;
    CflFluid fl[3];
    int magnetic;    // B planes start at ib
    int ib;
};

// timestep_fluid (src/base/timestep.F90:431-495) over the interior cells:
// per fluid, the maxima of c_d = max(|v_d| + c_s, small) for d = x, y, z and of
// max_d c_d.  Because dl/c is monotone in c under correct rounding,
// min_cells(dl/c_d) == dl/max_cells(c_d) exactly, so the host finishes the
// reduction with one division per direction.  Maxima of positive doubles are
// reduced as their bit patterns (order-independent, deterministic).
// out[f*4 + d] (d < 3) and out[f*4 + 3] hold the bit patterns.
// leaf (or null: every cell) marks the interior cells that no finer block
// covers (cg%leafmap, timestep.F90:463); the others are skipped.
PK_DEV void cfl_block(const BoxGeom& b, const double* __restrict__ u, const CflArgs& a, unsigned long long* __restrict__ out,
                      long long first, long long stride, const unsigned char* __restrict__ leaf = nullptr)
{
    const double small = 1.1754943508222875e-38;   // tiny(real(1.0,4)), constants.F90:104
    const long long ncell = (long long)b.n[0] * b.n[1] * b.n[2];
    double cm[3][4];
#pragma unroll
    for (int f = 0; f < 3; ++f)
#pragma unroll
        for (int d = 0; d < 4; ++d) cm[f][d] = small;
    const bool small_block = ncell <= 0x7fffffffLL;            // 32-bit index arithmetic suffices
    for (long long c = first; c < ncell; c += stride) {
        if (leaf && !leaf[c]) continue;
        int i, j, k;
        if (small_block) {
            const int ci = (int)c, r = ci / b.n[0];
            i = ci - r * b.n[0];
            j = r % b.n[1];
            k = r / b.n[1];
        } else {
            i = (int)(c % b.n[0]);
            const long long r = c / b.n[0];
            j = (int)(r % b.n[1]);
            k = (int)(r / b.n[1]);
        }
        const long long off = cell_index(b, i + b.g[0], j + b.g[1], k + b.g[2]);
        double pmag = 0.0;
        if (a.magnetic) {
            const double bx = u[(long long)(a.ib + 0) * b.plane + off];
            const double by = u[(long long)(a.ib + 1) * b.plane + off];
            const double bz = u[(long long)(a.ib + 2) * b.plane + off];
            pmag = 0.5 * ((bx * bx + by * by) + bz * bz);      // emag(b(x), b(y), b(z))
        }
#pragma unroll
        for (int f = 0; f < 3; ++f) {
            if (f >= a.nfl) break;
            const CflFluid fl = a.fl[f];
            const double dn = u[(long long)fl.beg * b.plane + off];
            const double mx = u[(long long)(fl.beg + 1) * b.plane + off];
            const double my = u[(long long)(fl.beg + 2) * b.plane + off];
            const double mz = u[(long long)(fl.beg + 3) * b.plane + off];
            double v[3];
            if (dn > 0.0) {                                     // timestep.F90:466-471
                v[0] = fabs(mx / dn);
                v[1] = fabs(my / dn);
                v[2] = fabs(mz / dn);
            } else {
                v[0] = v[1] = v[2] = 0.0;
            }
            double cs = 0.0;
            if (fl.kind != K_DST) {
                const double en = u[(long long)(fl.beg + 4) * b.plane + off];
                const double ek = (0.5 * ((mx * mx + my * my) + mz * mz)) / dn;
                if (fl.kind == K_ION) {                         // ion_cs, initionized.F90:131-139
                    const double ps = (en - ek) * fl.gam_1 + (2.0 - fl.gam) * pmag;
                    const double p = ps - pmag;
                    cs = sqrt(fabs((2.0 * pmag + fl.gam * p) / dn));
                } else {                                        // neu_cs, initneutral.F90:102-105
                    const double p = (en - ek) * fl.gam_1;
                    cs = sqrt(fabs((fl.gam * p) / dn));
                }
            }
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                const double cd = f_max(v[d] + cs, small);
                cm[f][d] = f_max(cm[f][d], cd);
                cm[f][3] = f_max(cm[f][3], cd);
            }
        }
    }
    __shared__ unsigned long long red[32][12];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int f = 0; f < 3; ++f)
#pragma unroll
        for (int d = 0; d < 4; ++d) {
            unsigned long long x = (unsigned long long)__double_as_longlong(cm[f][d]);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const unsigned long long y = __shfl_xor_sync(0xffffffffu, x, o);
                x = y > x ? y : x;
            }
            if (lane == 0) red[wid][f * 4 + d] = x;
        }
    __syncthreads();
    if (threadIdx.x < 12) {
        unsigned long long x = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) x = red[w][threadIdx.x] > x ? red[w][threadIdx.x] : x;
        atomicMax(out + threadIdx.x, x);
    }
}

// three CTAs of 256 threads per SM: the reduction is latency-bound (dependent
// division and square-root chains), so resident warps matter more than registers
static __global__ void __launch_bounds__(256, 3)
k_cfl(BoxGeom b, const double* __restrict__ u, CflArgs a, unsigned long long* __restrict__ out)
{
    cfl_block(b, u, a, out, (long long)blockIdx.x * blockDim.x + threadIdx.x, (long long)gridDim.x * blockDim.x);
}

// the same over a table of blocks: blockIdx.y picks the block, out has 12 slots per block
static __global__ void __launch_bounds__(256, 3)
k_cfl_blocks(const BlockDesc* __restrict__ blocks, CflArgs a, unsigned long long* __restrict__ out)
{
    const BlockDesc d = blocks[blockIdx.y];
    if ((long long)blockIdx.x * blockDim.x >= (long long)d.n[0] * d.n[1] * d.n[2]) return;   // CTAs a smaller block does not need
    BoxGeom b;
    for (int k = 0; k < 3; ++k) {
        b.ext[k] = d.ext[k];
        b.g[k] = d.g[k];
        b.n[k] = d.n[k];
    }
    b.plane = d.plane;
    cfl_block(b, d.in, a, out + 12 * blockIdx.y, (long long)blockIdx.x * blockDim.x + threadIdx.x,
              (long long)gridDim.x * blockDim.x, d.leaf);
}


// point_chspeed (hdc.F90:197-268): the gas-based GLM speed of one cell, from
// the first fluid of the set (ionized if present, else neutral, else dust),
// in the reference's operation order
struct ChArgs {
    int kind;                // K_ION / K_NEU / K_DST of fluid 0
    double gam, gam_1, cfl_glm;
    int has_dir[3];          // dom%has_dir
    int ib;                  // first B plane
};

PK_DEV double point_chspeed(const double* __restrict__ u, long long plane, long long off, const ChArgs& a)
{
    const double small = 1.1754943508222875e-38;        // constants.F90:104
    double ch = small;
    const double dn = u[off];
    const double m[3] = {u[plane + off], u[2 * plane + off], u[3 * plane + off]};
    if (a.kind == K_ION) {
        const double bx = u[(long long)a.ib * plane + off], by = u[(long long)(a.ib + 1) * plane + off],
                     bz = u[(long long)(a.ib + 2) * plane + off];
        const double bv[3] = {bx, by, bz};
        const double pmag = 0.5 * ((bx * bx + by * by) + bz * bz);                      // emag
        const double ek = (0.5 * ((m[0] * m[0] + m[1] * m[1]) + m[2] * m[2])) / dn;     // ekin
        const double pgam = ((0.5 * a.gam) * a.gam_1) * ((u[4 * plane + off] - ek) - pmag);
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            if (!a.has_dir[d]) continue;
            const double s = pgam + pmag;
            const double c = a.cfl_glm * (fabs(m[d] / dn) + sqrt((s + sqrt(s * s - (2.0 * pgam) * (bv[d] * bv[d]))) / dn));
            ch = f_max(ch, c);
        }
    } else if (a.kind == K_NEU) {
        const double ek = (0.5 * ((m[0] * m[0] + m[1] * m[1]) + m[2] * m[2])) / dn;
        const double pgam = ((0.5 * a.gam) * a.gam_1) * (u[4 * plane + off] - ek);
#pragma unroll
        for (int d = 0; d < 3; ++d)
            if (a.has_dir[d]) ch = f_max(ch, a.cfl_glm * (fabs(m[d] / dn) + sqrt((2.0 * pgam) / dn)));
    } else {
#pragma unroll
        for (int d = 0; d < 3; ++d)
            if (a.has_dir[d]) ch = f_max(ch, a.cfl_glm * fabs(m[d] / dn));
    }
    return ch;
}

// update_chspeed with ch_grid = .false. (hdc.F90:118-131): the maximum of
// point_chspeed over the interior leaf cells of every block (blockIdx.y picks
// the block), reduced as bit patterns of positive doubles into *out
static __global__ void __launch_bounds__(256, 3)
k_chspeed_blocks(const BlockDesc* __restrict__ blocks, ChArgs a, unsigned long long* __restrict__ out)
{
    const BlockDesc d = blocks[blockIdx.y];
    const long long ncell = (long long)d.n[0] * d.n[1] * d.n[2];
    unsigned long long best = 0;
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < ncell; c += (long long)gridDim.x * blockDim.x) {
        if (d.leaf && !d.leaf[c]) continue;
        const long long i = c % d.n[0], r = c / d.n[0];
        const long long j = r % d.n[1], k = r / d.n[1];
        const long long off = ((k + d.g[2]) * d.ext[1] + (j + d.g[1])) * d.ext[0] + (i + d.g[0]);
        const unsigned long long x = (unsigned long long)__double_as_longlong(point_chspeed(d.in, d.plane, off, a));
        best = x > best ? x : best;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long y = __shfl_xor_sync(0xffffffffu, best, o);
        best = y > best ? y : best;
    }
    if ((threadIdx.x & 31) == 0 && best) atomicMax(out, best);
}

// psi *= fac over the whole plane, guard cells included (hdc.F90:338)
static __global__ void k_scale(double* __restrict__ p, long long n, double fac)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        p[i] = p[i] * fac;
}

// the same for the step's factor in device memory (sp->psi_fac), over the
// psi plane (plane index ipsi) of every block of a table: blockIdx.y picks the block
static __global__ void k_scale_blocks(const BlockDesc* __restrict__ blocks, int ipsi,
                                      const StepParams* __restrict__ sp)
{
    const BlockDesc b = blocks[blockIdx.y];
    double* p = const_cast<double*>(b.in) + (long long)ipsi * b.plane;
    const double fac = sp->psi_fac;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < b.plane; i += (long long)gridDim.x * blockDim.x)
        p[i] = p[i] * fac;
}

static __global__ void k_scale_dev(double* __restrict__ p, long long n, const StepParams* __restrict__ sp)
{
    const double fac = sp->psi_fac;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        p[i] = p[i] * fac;
}

struct GuardArgs {
    int bnd[3][2];      // 0 per, 1 out, 2 ref
    int nplanes;
    int mom_plane[3][3];    // momentum planes per fluid and direction (-1: none)
    int nfl;
};

// Guard-cell refresh of one block, all components.  Filling x, then y over
// the x-extended range, then z (the order of the reference's per-direction
// exchanges) composes to: guard cell (i,j,k) takes the interior cell obtained
// by mapping each coordinate that lies in a guard layer through its boundary
// rule (periodic wrap, outflow clamp, reflecting mirror with the normal
// momentum negated) -- see bnd_u, src/grid/cg_list_bnd.F90:785-866.
__device__ __forceinline__ int map_guard(int i, int n, int g, int side_lo, int side_hi, bool& flip)
{
    if (i >= g && i < g + n) return i;
    if (i < g) {
        const int ib = g - i;                          // 1..g
        if (side_lo == 0) return g + n - ib;
        if (side_lo == 1) return g;
        flip = !flip;
        return g + ib - 1;
    }
    const int ib = i - (g + n - 1);                    // 1..g
    if (side_hi == 0) return g + ib - 1;
    if (side_hi == 1) return g + n - 1;
    flip = !flip;
    return g + n - ib;
}

static __global__ void k_fill_guards(BoxGeom b, double* __restrict__ u, GuardArgs a)
{
    const long long ncell = (long long)b.ext[0] * b.ext[1] * b.ext[2];
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < ncell; c += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(c % b.ext[0]);
        const long long r = c / b.ext[0];
        const int j = (int)(r % b.ext[1]);
        const int k = (int)(r / b.ext[1]);
        const bool inside = i >= b.g[0] && i < b.g[0] + b.n[0] && j >= b.g[1] && j < b.g[1] + b.n[1] &&
                            k >= b.g[2] && k < b.g[2] + b.n[2];
        if (inside) continue;
        bool fl[3] = {false, false, false};
        const int si = map_guard(i, b.n[0], b.g[0], a.bnd[0][0], a.bnd[0][1], fl[0]);
        const int sj = map_guard(j, b.n[1], b.g[1], a.bnd[1][0], a.bnd[1][1], fl[1]);
        const int sk = map_guard(k, b.n[2], b.g[2], a.bnd[2][0], a.bnd[2][1], fl[2]);
        const long long src = cell_index(b, si, sj, sk);
        for (int v = 0; v < a.nplanes; ++v) u[(long long)v * b.plane + c] = u[(long long)v * b.plane + src];
        for (int d = 0; d < 3; ++d)
            if (fl[d])
                for (int f = 0; f < a.nfl; ++f) {
                    const int pl = a.mom_plane[f][d];
                    u[(long long)pl * b.plane + c] = -u[(long long)pl * b.plane + c];
                }
    }
}

// Same-level guard exchange between blocks (cg_list_bnd.F90:286-314): one
// thread per guard cell of all segments; a segment is found by binary search
// over the running cell counts.  Sources are interior cells, targets guard
// cells, so the copies never race.
struct XSegDev {
    int dst, src;
    int lo[3], hi[3], shift[3];
    long long first;            // cells of all earlier segments
};

struct XPtr {
    double* u;
    long long plane;
    int ext[3];
};

// nplanes values from src (plane stride ss) to dst (stride ds), eight loads
// in flight before their stores (the two may alias as far as the compiler
// knows, which would otherwise serialise every load behind the last store)
PK_DEV void copy_planes(double* dst, long long ds, const double* src, long long ss, int nplanes)
{
    for (int v0 = 0; v0 < nplanes; v0 += 8) {
        double r[8];
#pragma unroll
        for (int k = 0; k < 8; ++k)
            if (v0 + k < nplanes) r[k] = src[(long long)(v0 + k) * ss];
#pragma unroll
        for (int k = 0; k < 8; ++k)
            if (v0 + k < nplanes) dst[(long long)(v0 + k) * ds] = r[k];
    }
}

// Same-level guard copies: each CTA takes whole segments (blockIdx.x, then
// every gridDim.x-th), its threads walk the segment's cells, i fastest.
static __global__ void k_exchange(const XSegDev* __restrict__ segs, int nseg, long long total,
                                  const XPtr* __restrict__ blk, int nplanes)
{
    (void)total;
    for (int sg = blockIdx.x; sg < nseg; sg += gridDim.x) {
        const XSegDev s = segs[sg];
        const int nx = s.hi[0] - s.lo[0], ny = s.hi[1] - s.lo[1], nz = s.hi[2] - s.lo[2];
        const long long cells = (long long)nx * ny * nz;
        const XPtr d = blk[s.dst], q = blk[s.src];
        for (long long r = threadIdx.x; r < cells; r += blockDim.x) {
            const int i = s.lo[0] + (int)(r % nx);
            const long long rr = r / nx;
            const int j = s.lo[1] + (int)(rr % ny);
            const int k = s.lo[2] + (int)(rr / ny);
            const long long di = ((long long)k * d.ext[1] + j) * d.ext[0] + i;
            const long long si =
                ((long long)(k + s.shift[2]) * q.ext[1] + (j + s.shift[1])) * q.ext[0] + (i + s.shift[0]);
            copy_planes(d.u + di, d.plane, q.u + si, q.plane, nplanes);
        }
    }
}

// Halo exchange with another rank: pack the source cells of the segments
// sent to one peer (to_buf = 1) or unpack the cells received from it into
// guard cells (to_buf = 0).  Buffer layout: plane v of cell c at v*total + c,
// cells in segment order, i fastest within a segment.
static __global__ void k_halo_copy(const XSegDev* __restrict__ segs, int nseg, long long total,
                                   const XPtr* __restrict__ blk, int nplanes, double* __restrict__ buf, int to_buf)
{
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < total; c += (long long)gridDim.x * blockDim.x) {
        int lo = 0, hi = nseg - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (segs[mid].first <= c) lo = mid;
            else hi = mid - 1;
        }
        const XSegDev s = segs[lo];
        long long r = c - s.first;
        const int nx = s.hi[0] - s.lo[0], ny = s.hi[1] - s.lo[1];
        const int i = s.lo[0] + (int)(r % nx);
        r /= nx;
        const int j = s.lo[1] + (int)(r % ny);
        const int k = s.lo[2] + (int)(r / ny);
        if (to_buf) {
            const XPtr q = blk[s.src];
            const long long si = ((long long)(k + s.shift[2]) * q.ext[1] + (j + s.shift[1])) * q.ext[0] + (i + s.shift[0]);
            copy_planes(buf + c, total, q.u + si, q.plane, nplanes);
        } else {
            const XPtr d = blk[s.dst];
            const long long di = ((long long)k * d.ext[1] + j) * d.ext[0] + i;
            copy_planes(d.u + di, d.plane, buf + c, total, nplanes);
        }
    }
}

// zero every guard cell of all planes (adjoint states carry no guard values)
static __global__ void k_zero_guards(BoxGeom b, double* __restrict__ u, int nplanes)
{
    const long long ncell = (long long)b.ext[0] * b.ext[1] * b.ext[2];
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < ncell; c += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(c % b.ext[0]);
        const long long r = c / b.ext[0];
        const int j = (int)(r % b.ext[1]);
        const int k = (int)(r / b.ext[1]);
        const bool inside = i >= b.g[0] && i < b.g[0] + b.n[0] && j >= b.g[1] && j < b.g[1] + b.n[1] &&
                            k >= b.g[2] && k < b.g[2] + b.n[2];
        if (!inside)
            for (int v = 0; v < nplanes; ++v) u[(long long)v * b.plane + c] = 0.0;
    }
}

// Fortran-order arrays (u(nvar,i,j,k), b(3,i,j,k), psi(i,j,k)) <-> component planes.
static __global__ void k_aos_to_soa(const double* __restrict__ aos, double* __restrict__ soa, long long ncell, int ncomp,
                             int plane0, long long plane)
{
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < ncell; c += (long long)gridDim.x * blockDim.x)
        for (int v = 0; v < ncomp; ++v) soa[(long long)(plane0 + v) * plane + c] = aos[c * ncomp + v];
}

static __global__ void k_soa_to_aos(const double* __restrict__ soa, double* __restrict__ aos, long long ncell, int ncomp,
                             int plane0, long long plane)
{
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < ncell; c += (long long)gridDim.x * blockDim.x)
        for (int v = 0; v < ncomp; ++v) aos[c * ncomp + v] = soa[(long long)(plane0 + v) * plane + c];
}

// copy the pencils a stage touched (full extent along dir, interior in the
// other two directions) from src to dst, all planes
static __global__ void k_copy_pencils(BoxGeom b, int dir, const double* __restrict__ src, double* __restrict__ dst, int nplanes)
{
    int lo[3], hi[3];
    for (int d = 0; d < 3; ++d) {
        lo[d] = (d == dir) ? 0 : b.g[d];
        hi[d] = (d == dir) ? b.ext[d] : b.g[d] + b.n[d];
    }
    const long long nx = hi[0] - lo[0], ny = hi[1] - lo[1], nz = hi[2] - lo[2];
    const long long ncell = nx * ny * nz;
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < ncell; c += (long long)gridDim.x * blockDim.x) {
        const int i = lo[0] + (int)(c % nx);
        const long long r = c / nx;
        const int j = lo[1] + (int)(r % ny);
        const int k = lo[2] + (int)(r / ny);
        const long long o = cell_index(b, i, j, k);
        for (int v = 0; v < nplanes; ++v) dst[(long long)v * b.plane + o] = src[(long long)v * b.plane + o];
    }
}

// ---- refined domains -------------------------------------------------------

// The fine->coarse flux sum of send_cg_coarsebnd (fc_fluxes.F90:213-225): each
// coarse face takes 0 + the fine faces' fluxes in the reference's loop order
// (ORTHO1 outer, ORTHO2 inner), times 1 / 2**(eff_dim - 1).
// ---------------------------------------------------------------------------
// E-GLM sources (hdc.F90:355-457; use_eglm, off by default, global.F90:252),
// applied after each triple of sweeps, before glmdamping, to the ionized
// fluid of one block whose guard cells are current.  k_eglm_grad stores, for
// every interior cell, divB of order 2 (divB.F90:146-249: coeff_c(1) = 1/2
// times the sum over directions of (b(+1) - b(-1)) / dl, sixpoint :297-338)
// and grad(psi) = (1/2 (psi(+1) - psi(-1))) / dl (:396-401) in w (4 planes of
// the block's plane size) before any cell changes; k_eglm_apply then updates
// each interior cell in the reference's statement order (:414-432), every
// line using the previous lines' results:
//   m -= (dt divB) B;  B -= (dt divB) (m/rho);
//   E -= dt (divB (m/rho).B - B.grad(psi));  psi -= dt (m/rho).grad(psi)
// with dot products accumulated from zero as dot_product does.  A direction
// of extent 1 (D = 0) contributes (b - b) / dl = 0.
// ---------------------------------------------------------------------------
struct EglmArgs {
    int n[3], g[3], ext[3];
    int D[3];               // 1 where the direction has more than one cell (dom%D_x, D_y, D_z)
    long long plane;
    double dl[3];
    int ib;                 // first B plane; psi is plane ib + 3
    int idn;                // the ionized fluid's density plane (momenta idn+1..3, energy idn+4); -1 none
};

PK_DEV long long eglm_cell(const EglmArgs& a, long long c)
{
    const int i = (int)(c % a.n[0]) + a.g[0];
    const long long r = c / a.n[0];
    const int j = (int)(r % a.n[1]) + a.g[1];
    const int k = (int)(r / a.n[1]) + a.g[2];
    return (long long)i + (long long)j * a.ext[0] + (long long)k * a.ext[0] * a.ext[1];
}

static __global__ void k_eglm_grad(const double* __restrict__ u, double* __restrict__ w, EglmArgs a)
{
    const long long ncell = (long long)a.n[0] * a.n[1] * a.n[2];
    const long long st[3] = {1, a.ext[0], (long long)a.ext[0] * a.ext[1]};
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < ncell;
         c += (long long)gridDim.x * blockDim.x) {
        const long long s = eglm_cell(a, c);
        double t[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const long long sp = s + a.D[d] * st[d], sm = s - a.D[d] * st[d];
            const double* bd = u + (long long)(a.ib + d) * a.plane;
            const double* ps = u + (long long)(a.ib + 3) * a.plane;
            t[d] = (bd[sp] - bd[sm]) / a.dl[d];
            w[(long long)(1 + d) * a.plane + s] = (0.5 * (ps[sp] - ps[sm])) / a.dl[d];
        }
        w[s] = 0.5 * ((t[0] + t[1]) + t[2]);
    }
}

static __global__ void k_eglm_apply(double* __restrict__ u, const double* __restrict__ w, EglmArgs a,
                                    const StepParams* __restrict__ sp)
{
    const double dt = sp->dt;
    const long long ncell = (long long)a.n[0] * a.n[1] * a.n[2];
    const long long P = a.plane;
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < ncell;
         c += (long long)gridDim.x * blockDim.x) {
        const long long s = eglm_cell(a, c);
        const double q = w[s], dq = dt * q;
        const double gp[3] = {w[P + s], w[2 * P + s], w[3 * P + s]};
        const double rho = u[(long long)a.idn * P + s];
        double m[3], B[3], v[3];
#pragma unroll
        for (int c3 = 0; c3 < 3; ++c3) {
            m[c3] = u[(long long)(a.idn + 1 + c3) * P + s] - dq * u[(long long)(a.ib + c3) * P + s];
            v[c3] = m[c3] / rho;
            B[c3] = u[(long long)(a.ib + c3) * P + s] - dq * v[c3];
        }
        const double vb = ((0.0 + v[0] * B[0]) + v[1] * B[1]) + v[2] * B[2];
        const double bg = ((0.0 + B[0] * gp[0]) + B[1] * gp[1]) + B[2] * gp[2];
        const double vg = ((0.0 + v[0] * gp[0]) + v[1] * gp[1]) + v[2] * gp[2];
        double* e = u + (long long)(a.idn + 4) * P + s;
        *e = *e - dt * (q * vb - bg);
        double* ps = u + (long long)(a.ib + 3) * P + s;
        *ps = *ps - dt * vg;
#pragma unroll
        for (int c3 = 0; c3 < 3; ++c3) {
            u[(long long)(a.idn + 1 + c3) * P + s] = m[c3];
            u[(long long)(a.ib + c3) * P + s] = B[c3];
        }
    }
}

static __global__ void k_restrict_flux(const int* __restrict__ src, int beg, int end, int nv,
                                       const double* __restrict__ out_flux, double* __restrict__ in_flux, double scale)
{
    const long long n = (long long)(end - beg) * nv;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int slot = beg + (int)(t / nv);
        const int v = (int)(t % nv);
        double acc = 0.0;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int s = src[4 * slot + q];
            if (s >= 0) acc = acc + out_flux[(long long)s * nv + v];
        }
        in_flux[(long long)slot * nv + v] = scale * acc;
    }
}

struct PRunDev {
    int fb, cb;
    int fx, fy, fz, len;
    int cx, cy, cz;
    int px, py, pz;
};

// The directional stencil of one prolongation order
// (grid_container_prolong.F90:180-453): coefficients P_3..P3 in p[0..6] and
// the stencil range r (0: injection).
struct ProlongCoef {
    double p[7];
    int r;
};

// one centred interpolation along a direction: the left child (par 0) takes
// sum over m = -r..r of P(-m) c(m), the right child sum of P(m) c(m), added
// left to right in increasing m; c points at the parent, s is the stride
PK_DEV double prolong_1d(const ProlongCoef& k, const double* c, long long s, int par)
{
    if (k.r == 0) return c[0];
    double acc = 0.0;
    for (int m = -k.r; m <= k.r; ++m) {
        const double t = k.p[3 + (par == 0 ? -m : m)] * c[m * s];
        acc = (m == -k.r) ? t : acc + t;
    }
    return acc;
}

// prolong_bnd_from_coarser (cg_level_connected.F90:1150-1359) for the guard
// cells of one level: the fluid planes with the stencil ku (ord_fluid_prolong),
// B and psi with kb (ord_mag_prolong), each split by direction as prolong()
// does: x over the (2r+1)^2 coarse rows around the parent, then y, then z.
// runs has nruns rows; start[r] is the running cell count before run r.
PK_DEV double prolong_cell(const ProlongCoef& k, const double* c, long long sx, long long sy, long long sz, int px,
                           int py, int pz, bool hx, bool hy, bool hz)
{
    const int ry = hy ? k.r : 0, rz = hz ? k.r : 0;
    double Y[7];
    for (int kz = -rz; kz <= rz; ++kz) {
        double X[7];
        for (int ky = -ry; ky <= ry; ++ky) {
            const double* row = c + ky * sy + kz * sz;
            X[ky + 3] = hx ? prolong_1d(k, row, sx, px) : row[0];
        }
        Y[kz + 3] = hy ? prolong_1d(k, X + 3, 1, py) : X[3];
    }
    return hz ? prolong_1d(k, Y + 3, 1, pz) : Y[3];
}

static __global__ void k_prolong(const PRunDev* __restrict__ runs, const long long* __restrict__ start, int nruns,
                                 long long total, const XPtr* __restrict__ blocks, int nu, int nmag, int has_x,
                                 int has_y, int has_z, ProlongCoef ku, ProlongCoef kb, ProlongCoef kpsi)
{
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
        int lo = 0, hi = nruns - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (start[mid] <= t) lo = mid;
            else hi = mid - 1;
        }
        const PRunDev r = runs[lo];
        const int i = (int)(t - start[lo]);
        const XPtr F = blocks[r.fb], C = blocks[r.cb];
        const int px = (r.px + i) & 1;
        const int cx = r.cx + ((r.px + i) >> 1);
        const long long fo = ((long long)r.fz * F.ext[1] + r.fy) * F.ext[0] + (r.fx + i);
        const long long co = ((long long)r.cz * C.ext[1] + r.cy) * C.ext[0] + cx;
        const long long sx = has_x, sy = has_y ? C.ext[0] : 0, sz = has_z ? (long long)C.ext[0] * C.ext[1] : 0;
        if (ku.r == 0) {
            copy_planes(F.u + fo, F.plane, C.u + co, C.plane, nu);   // O_INJ
        } else {
            for (int v = 0; v < nu; ++v)
                F.u[(long long)v * F.plane + fo] = prolong_cell(ku, C.u + (long long)v * C.plane + co, sx, sy, sz, px,
                                                                r.py, r.pz, has_x, has_y, has_z);
        }
        for (int v = nu; v < nu + nmag; ++v)
            F.u[(long long)v * F.plane + fo] = prolong_cell(v < nu + 3 ? kb : kpsi, C.u + (long long)v * C.plane + co, sx,
                                                            sy, sz, px, r.py, r.pz, has_x, has_y, has_z);
    }
}

// apply_flux, update_psi and apply_source of one stage (solve_cg_unsplit.F90:
// 167-229, unsplit_mag_modules.F90:195-350, unsplit_source.F90:36-132), one
// thread per cell of the guard-inclusive block.  T starts as S (the first
// RK2 stage writes the copy uh = u: S = u, T = uh; otherwise S = T = u) and
// gains, for d = x, y, z over
// bounds_for_flux(d) (every cell but the outermost layer along d, interior
// across), (dt / dl(d)) * rk * (F_d(i) - F_d(i+1)); every plane, B and psi
// included.  Then each cell on an interior pencil of direction d (d = x, y,
// z with extent) gets internal_sources (+0) and, at the last stage,
// care_for_positives in d's swept component order, once per such d.
template <class PH>
__global__ void k_unsplit_apply(BoxGeom b, const double* S, double* T,
                                const double* __restrict__ Fx, const double* __restrict__ Fy,
                                const double* __restrict__ Fz, PhysParams pp, const StepParams* __restrict__ spar,
                                double rk, double dlx, double dly, double dlz, int last, unsigned* __restrict__ gstatus)
{
    constexpr int NV = PH::NV;
    unsigned status = 0;
    const long long ncell = (long long)b.ext[0] * b.ext[1] * b.ext[2];
    const double* Fd[3] = {Fx, Fy, Fz};
    const double dl[3] = {dlx, dly, dlz};
    const long long stride[3] = {1, b.ext[0], (long long)b.ext[0] * b.ext[1]};
    const double dt = spar->dt;
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < ncell; c += (long long)gridDim.x * blockDim.x) {
        int x[3];
        x[0] = (int)(c % b.ext[0]);
        const long long rr = c / b.ext[0];
        x[1] = (int)(rr % b.ext[1]);
        x[2] = (int)(rr / b.ext[1]);
        bool in[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) in[d] = b.n[d] <= 1 || (x[d] >= b.g[d] && x[d] < b.g[d] + b.n[d]);
        double nat[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) nat[v] = S[(long long)v * b.plane + c];
#pragma unroll
        for (int af = 0; af < 3; ++af) {
            if (b.n[af] <= 1) continue;
            bool reg = x[af] >= 1 && x[af] <= b.ext[af] - 2;
#pragma unroll
            for (int d = 0; d < 3; ++d)
                if (d != af) reg = reg && in[d];
            if (!reg) continue;
            const double coef = (dt / dl[af]) * rk;
            const double* F = Fd[af];
#pragma unroll
            for (int v = 0; v < NV; ++v)
                nat[v] = nat[v] + coef * (F[(long long)v * b.plane + c] - F[(long long)v * b.plane + c + stride[af]]);
        }
#pragma unroll
        for (int dd = 0; dd < 3; ++dd) {
            if (b.n[dd] <= 1) continue;
            bool pencil = true;                       // on a pencil of dd through the interior
#pragma unroll
            for (int d = 0; d < 3; ++d)
                if (d != dd) pencil = pencil && in[d];
            if (!pencil) continue;
            if (!last) {
#pragma unroll
                for (int v = 0; v < PH::NVF; ++v) nat[v] = nat[v] + 0.0;
                continue;
            }
            const int perm[3] = {dd, dd == 1 ? 0 : 1, dd == 2 ? 0 : 2};   // iarr_swp of dd
            double w[NV];
#pragma unroll
            for (int v = 0; v < NV; ++v) w[v] = nat[plane_of<PH>(v, perm)];
            sources_and_floors<PH>(w, pp, status);
#pragma unroll
            for (int v = 0; v < NV; ++v) nat[plane_of<PH>(v, perm)] = w[v];
        }
#pragma unroll
        for (int v = 0; v < NV; ++v) T[(long long)v * b.plane + c] = nat[v];
    }
    flush_status(status, gstatus);
}

struct RBoxDev {
    int fb, cb;
    int lo[3], hi[3], flo[3];
};

// restrict (cg_level_connected.F90:1480-1721) of one level into the next
// coarser one: each covered coarse cell takes the mean of its children, every
// plane.  With three directions the eight children are summed x fastest and
// scaled once (the even-offset array form, :1566-1590); with fewer, each
// child is scaled and accumulated from 0 in z, y, x loop order (:1613-1631).
// The coarse cell then becomes 0 + that (:1654-1680).
static __global__ void k_restrict(const RBoxDev* __restrict__ boxes, const long long* __restrict__ start, int nbox,
                                  long long total, const XPtr* __restrict__ blocks, int nplanes, int has_x, int has_y,
                                  int has_z, double norm)
{
    const bool full3 = has_x && has_y && has_z;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
        int lo = 0, hi = nbox - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (start[mid] <= t) lo = mid;
            else hi = mid - 1;
        }
        const RBoxDev bx = boxes[lo];
        long long r = t - start[lo];
        const int nx = bx.hi[0] - bx.lo[0], ny = bx.hi[1] - bx.lo[1];
        const int i = (int)(r % nx);
        r /= nx;
        const int j = (int)(r % ny);
        const int k = (int)(r / ny);
        const XPtr C = blocks[bx.cb], F = blocks[bx.fb];
        const long long co = ((long long)(bx.lo[2] + k) * C.ext[1] + (bx.lo[1] + j)) * C.ext[0] + (bx.lo[0] + i);
        const int fx = bx.flo[0] + (has_x ? 2 * i : 0), fy = bx.flo[1] + (has_y ? 2 * j : 0),
                  fz = bx.flo[2] + (has_z ? 2 * k : 0);
        const long long sx = 1, sy = F.ext[0], sz = (long long)F.ext[0] * F.ext[1];
        const long long fo = fz * sz + fy * sy + fx;
        for (int v = 0; v < nplanes; ++v) {
            const double* f = F.u + (long long)v * F.plane + fo;
            double val;
            if (full3) {
                val = (((((((f[0] + f[sx]) + f[sy]) + f[sx + sy]) + f[sz]) + f[sx + sz]) + f[sy + sz]) + f[sx + sy + sz]) *
                      norm;
            } else {
                double acc = 0.0;
                for (int kz = 0; kz <= has_z; ++kz)
                    for (int jy = 0; jy <= has_y; ++jy)
                        for (int ix = 0; ix <= has_x; ++ix) acc = acc + f[kz * sz + jy * sy + ix * sx] * norm;
                val = acc;
            }
            C.u[(long long)v * C.plane + co] = 0.0 + val;
        }
    }
}

// ---------------------------------------------------------------------------
// Refinement criteria (URC_var.F90): one thread per guard-inclusive cell of
// each marked block sets the cell's flag when any criterion fires there.
// ---------------------------------------------------------------------------
struct UrcDev {
    int method, field;
    double thr, aux;
};

struct MarkBlk {
    const double* u;
    long long plane;
    int ext[3], g[3], n[3];
    int level;
    double idl[3];                  // 1 / dl (cg%idl)
    unsigned char* map;             // ext cells, x fastest
    const unsigned char* leaf;      // interior leaf mask or null (all leaf)
};

// first differences of refine_on_second_derivative (URC_var.F90:447-505):
// du = (p(+1) - p(-1)) * idl, dau = (|p(+1)| + |p(-1)|) * idl along stride s
PK_DEV double urc_du(const double* p, long long s, double id) { return (p[s] - p[-s]) * id; }
PK_DEV double urc_dau(const double* p, long long s, double id) { return (fabs(p[s]) + fabs(p[-s])) * id; }

// one cross term of the Loechner denominator: ((|du(+t)| + |du(-t)|) + aux (dau(+t) + dau(-t))) * id_t,
// du and dau taken along s and evaluated at the neighbours along t
PK_DEV double urc_den(const double* p, long long s, double ids, long long t, double idt, double aux)
{
    return ((fabs(urc_du(p + t, s, ids)) + fabs(urc_du(p - t, s, ids))) +
            aux * (urc_dau(p + t, s, ids) + urc_dau(p - t, s, ids))) * idt;
}

// Loechner's estimator (refine_on_second_derivative, URC_var.F90:348-437)
PK_DEV double urc_loechner(const double* p, const long long st[3], const double id[3], const bool has[3], double aux)
{
    double sn = 0.0, sd = 0.0;
    if (has[0]) {
        double t = (urc_du(p + st[0], st[0], id[0]) - urc_du(p - st[0], st[0], id[0])) * id[0];
        double a = urc_den(p, st[0], id[0], st[0], id[0], aux);
        sn = sn + t * t;
        sd = sd + a * a;
        if (has[1]) {
            t = (urc_du(p + st[1], st[0], id[0]) - urc_du(p - st[1], st[0], id[0])) * id[1];
            sn = sn + 2.0 * (t * t);
            a = urc_den(p, st[0], id[0], st[1], id[1], aux);
            const double b = urc_den(p, st[1], id[1], st[0], id[0], aux);
            sd = (sd + a * a) + b * b;
        }
        if (has[2]) {
            t = (urc_du(p + st[2], st[0], id[0]) - urc_du(p - st[2], st[0], id[0])) * id[2];
            sn = sn + 2.0 * (t * t);
            a = urc_den(p, st[0], id[0], st[2], id[2], aux);
            const double b = urc_den(p, st[2], id[2], st[0], id[0], aux);
            sd = (sd + a * a) + b * b;
        }
    }
    if (has[1]) {
        double t = (urc_du(p + st[1], st[1], id[1]) - urc_du(p - st[1], st[1], id[1])) * id[1];
        double a = urc_den(p, st[1], id[1], st[1], id[1], aux);
        sn = sn + t * t;
        sd = sd + a * a;
        if (has[2]) {
            t = (urc_du(p + st[2], st[1], id[1]) - urc_du(p - st[2], st[1], id[1])) * id[2];
            sn = sn + 2.0 * (t * t);
            a = urc_den(p, st[1], id[1], st[2], id[2], aux);
            const double b = urc_den(p, st[2], id[2], st[1], id[1], aux);
            sd = (sd + a * a) + b * b;
        }
    }
    if (has[2]) {
        const double t = (urc_du(p + st[2], st[2], id[2]) - urc_du(p - st[2], st[2], id[2])) * id[2];
        const double a = urc_den(p, st[2], id[2], st[2], id[2], aux);
        sn = sn + t * t;
        sd = sd + a * a;
    }
    if (sd > 0.0) return sn / sd;
    return sn > 0.0 ? 1.0 : 0.0;
}

// |a - b| / (|a| + |b|), 0 when either is 0 (rel_grad_1pair, URC_var.F90:674-688)
PK_DEV double urc_rel1(double a, double b)
{
    if (fabs(a) != 0.0 && fabs(b) != 0.0) return fabs(a - b) / (fabs(a) + fabs(b));
    return 0.0;
}

// a (+) b squared (sumsq01, URC_var.F90:690-706)
PK_DEV double urc_sumsq01(double a, double b) { return (a * a) * (1.0 - b * b) + b * b; }

static __global__ void k_mark(const MarkBlk* __restrict__ blks, const long long* __restrict__ start, int nblk,
                              long long total, const UrcDev* __restrict__ crit, int ncrit, int hx, int hy, int hz,
                              int* __restrict__ flagged)
{
    const bool has[3] = {hx != 0, hy != 0, hz != 0};
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
        int lo = 0, hi = nblk - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (start[mid] <= t) lo = mid;
            else hi = mid - 1;
        }
        const MarkBlk B = blks[lo];
        long long r = t - start[lo];
        const int x = (int)(r % B.ext[0]);
        r /= B.ext[0];
        const int y = (int)(r % B.ext[1]);
        const int z = (int)(r / B.ext[1]);
        const int ic[3] = {x - B.g[0], y - B.g[1], z - B.g[2]};
        bool inside = true, near = true;          // interior; interior widened by 2 along each direction with extent
        for (int d = 0; d < 3; ++d) {
            inside = inside && ic[d] >= 0 && ic[d] < B.n[d];
            const int w = has[d] ? 2 : 0;
            near = near && ic[d] >= -w && ic[d] < B.n[d] + w;
        }
        const long long cell = ((long long)z * B.ext[1] + y) * B.ext[0] + x;
        const long long st[3] = {has[0] ? 1 : 0, has[1] ? (long long)B.ext[0] : 0,
                                 has[2] ? (long long)B.ext[0] * B.ext[1] : 0};
        unsigned char f = 0;
        for (int c = 0; c < ncrit; ++c) {
            const UrcDev C = crit[c];
            const double* p = B.u + (long long)C.field * B.plane + cell;
            if (C.method == PK_URC_LOECHNER) {
                if (near && urc_loechner(p, st, B.idl, has, C.aux) >= C.thr) f = 1;
                continue;
            }
            if (!inside) continue;
            if (C.method == PK_URC_THRESHOLD) {
                if (C.aux > 0.0 && (double)B.level >= C.aux) continue;
                if (p[0] >= C.thr) f = 1;
            } else if (C.method == PK_URC_GRAD) {
                const double a = p[st[0]] - p[-st[0]], b = p[st[1]] - p[-st[1]], e = p[st[2]] - p[-st[2]];
                if ((a * a + b * b) + e * e >= C.thr * C.thr) f = 1;
            } else if (C.method == PK_URC_RELGRAD) {
                double g2 = 0.0;
                if (has[0]) g2 = urc_sumsq01(urc_rel1(p[0], p[st[0]]), urc_rel1(p[0], p[-st[0]]));
                if (has[1]) g2 = urc_sumsq01(g2, urc_sumsq01(urc_rel1(p[0], p[st[1]]), urc_rel1(p[0], p[-st[1]])));
                if (has[2]) g2 = urc_sumsq01(g2, urc_sumsq01(urc_rel1(p[0], p[st[2]]), urc_rel1(p[0], p[-st[2]])));
                if (g2 >= C.thr * C.thr) f = 1;
            }
        }
        B.map[cell] = f;
        if (f && inside && (!B.leaf || B.leaf[((long long)ic[2] * B.n[1] + ic[1]) * B.n[0] + ic[0]])) flagged[lo] = 1;
    }
}

}  // namespace pk
