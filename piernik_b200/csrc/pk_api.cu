// pk_api.cu -- C ABI of libpiernik_b200.so: block registry, host<->device
// layout conversion, kernel dispatch and the host-side time-step logic of
// PIERNIK's main loop for the split Riemann path.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "pk_aux.cuh"
#include "pk_exchange.h"
#include "pk_internal.h"

using namespace pk;

namespace pk {

int fail(pk_ctx* h, int code, const std::string& msg)
{
    h->err = msg;
    return code;
}

int ev_begin(pk_ctx* h, std::pair<cudaEvent_t, cudaEvent_t>* p)
{
    if (!h->profiling) return PK_OK;
    if (h->ev_free.empty()) {
        cudaEvent_t a, b;
        if (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess) return PK_E_CUDA;
        h->ev_free.push_back({a, b});
    }
    *p = h->ev_free.back();
    h->ev_free.pop_back();
    if (cudaEventRecord(p->first, h->stream) != cudaSuccess) return PK_E_CUDA;
    return PK_OK;
}

int ev_end(pk_ctx* h, const std::pair<cudaEvent_t, cudaEvent_t>& p)
{
    if (!h->profiling) return PK_OK;
    if (cudaEventRecord(p.second, h->stream) != cudaSuccess) return PK_E_CUDA;
    h->ev_used.push_back(p);
    return PK_OK;
}

// ORTHO pairs with the memory-fastest ortho direction first (lanes/coalescing)
static constexpr int ORTHO1[3] = {1, 0, 0};
static constexpr int ORTHO2[3] = {2, 2, 1};
static constexpr int PERM3[3][3] = {{0, 1, 2}, {1, 0, 2}, {2, 1, 0}};

Geom make_geom(const Block& b, int dir)
{
    Geom g;
    const long long st[3] = {1, b.ext[0], (long long)b.ext[0] * b.ext[1]};
    const int o1 = ORTHO1[dir], o2 = ORTHO2[dir];
    g.plane = b.plane;
    g.sd = st[dir];
    g.s1 = st[o1];
    g.s2 = st[o2];
    g.ext_d = b.ext[dir];
    g.n_d = b.n[dir];
    g.g_d = b.g[dir];
    g.n1 = b.n[o1];
    g.g1 = b.g[o1];
    g.n2 = b.n[o2];
    g.g2 = b.g[o2];
    for (int j = 0; j < 3; ++j) g.perm[j] = PERM3[dir][j];
    g.seg_len = b.seg_len;
    g.seg_along = dir == 2;
    return g;
}

}  // namespace pk

namespace {

int grid1d(long long n, int threads)
{
    long long b = (n + threads - 1) / threads;
    if (b > grid_cap()) b = grid_cap();
    return (int)(b < 1 ? 1 : b);
}

const FastOps* fast_ops_of(pk_ctx* h)
{
    switch (h->phys) {
    case 0: return fast_ops_hd1();
    case 1: return fast_ops_hd2();
    case 2: return fast_ops_mhd1();
    case 3: return fast_ops_mhd2();
    default: return fast_ops_mhd3();
    }
}

const PhysOps* ops_of(pk_ctx* h)
{
    switch (h->phys) {
    case 0: return ops_hd1();
    case 1: return ops_hd2();
    case 2: return ops_mhd1();
    case 3: return ops_mhd2();
    default: return ops_mhd3();
    }
}

BoxGeom box_of(const Block& b)
{
    BoxGeom bg;
    for (int d = 0; d < 3; ++d) {
        bg.ext[d] = b.ext[d];
        bg.g[d] = b.g[d];
        bg.n[d] = b.n[d];
    }
    bg.plane = b.plane;
    return bg;
}

double* state(pk_ctx* h, Block& b) { return b.buf[h->cur]; }

int fill_guards_ptr(pk_ctx* h, Block& b, double* u);

int fill_guards_block(pk_ctx* h, Block& b)
{
    if (int rc = fill_guards_ptr(h, b, state(h, b))) return rc;
    b.guards_stale = false;
    return PK_OK;
}

// update_boundaries of one block's own boundary rules on the array u
int fill_guards_ptr(pk_ctx* h, Block& b, double* u)
{
    GuardArgs a;
    int beg = 0;
    for (int d = 0; d < 3; ++d)
        for (int s = 0; s < 2; ++s) a.bnd[d][s] = b.bnd[d][s];
    for (int i = 0; i < 3; ++i)
        for (int d = 0; d < 3; ++d) a.mom_plane[i][d] = -1;
    for (int f = 0; f < h->cfg.nfluids; ++f) {
        for (int d = 0; d < 3; ++d) a.mom_plane[f][d] = beg + 1 + d;
        beg += (h->cfg.fluid_kind[f] == PK_FLUID_DST) ? 4 : 5;
    }
    a.nfl = h->cfg.nfluids;
    a.nplanes = h->nplanes;
    k_fill_guards<<<grid1d(b.plane, 256), 256, 0, h->stream>>>(box_of(b), u, a);
    PK_CUDA(h, cudaGetLastError());
    h->launches += 1;
    return PK_OK;
}

// Same-level exchange of all placed blocks' guard cells (update_boundaries'
// internal part); blocks' own boundary rules were applied before.  The plan
// and the per-parity block tables are built here, outside any graph capture.
int ensure_pingpong(pk_ctx* h);

int upload_segs(pk_ctx* h, const std::vector<XSeg>& segs, XSegList* out)
{
    std::vector<XSegDev> dev(segs.size());
    long long total = 0;
    for (size_t s = 0; s < segs.size(); ++s) {
        XSegDev& d = dev[s];
        d.dst = segs[s].dst;
        d.src = segs[s].src;
        long long cells = 1;
        for (int k = 0; k < 3; ++k) {
            d.lo[k] = segs[s].lo[k];
            d.hi[k] = segs[s].hi[k];
            d.shift[k] = segs[s].shift[k];
            cells *= segs[s].hi[k] - segs[s].lo[k];
        }
        d.first = total;
        total += cells;
    }
    cudaFree(out->dev);
    out->dev = nullptr;
    if (!dev.empty()) {
        PK_CUDA(h, cudaMalloc(&out->dev, sizeof(XSegDev) * dev.size()));
        PK_CUDA(h, cudaMemcpy(out->dev, dev.data(), sizeof(XSegDev) * dev.size(), cudaMemcpyHostToDevice));
    }
    out->n = (int)dev.size();
    out->total = total;
    return PK_OK;
}

void free_segs(pk_ctx* h)
{
    cudaFree(h->xlocal.dev);
    h->xlocal = XSegList();
    for (int d = 0; d < 3; ++d) {
        cudaFree(h->xlocal_dir[d].dev);
        h->xlocal_dir[d] = XSegList();
    }
    h->x_dir = false;
    for (auto& p : h->xpeers) {
        cudaFree(p.send.dev);
        cudaFree(p.recv.dev);
        for (int d = 0; d < 3; ++d) {
            cudaFree(p.send_dir[d].dev);
            cudaFree(p.recv_dir[d].dev);
        }
    }
    h->xpeers.clear();
}

// the segments of face boxes along dir (seg_face_dir of their destination block)
static std::vector<XSeg> face_segs(const std::vector<XBlock>& xb, const std::vector<XSeg>& segs, int dir)
{
    std::vector<XSeg> out;
    for (const XSeg& s : segs)
        if (seg_face_dir(xb[s.dst], s) == dir) out.push_back(s);
    return out;
}

void free_levels(pk_ctx* h)
{
    for (auto& q : h->part) {
        cudaFree(q.segs.dev);
        cudaFree(q.runs);
        cudaFree(q.run_start);
        q = pk_ctx::Partial();
    }
    cudaFree(h->d_rbox);
    cudaFree(h->d_rbox_start);
    h->d_rbox = nullptr;
    h->d_rbox_start = nullptr;
    h->rbox_beg.clear();
    h->rbox_cells.clear();
    cudaFree(h->d_runs);
    cudaFree(h->d_run_start);
    h->d_runs = nullptr;
    h->d_run_start = nullptr;
    h->run_beg.clear();
    h->run_cells.clear();
    for (int d = 0; d < 3; ++d) {
        cudaFree(h->d_fc_int[d]);
        cudaFree(h->d_in_flux[d]);
        cudaFree(h->d_out_flux[d]);
        h->d_fc_int[d] = nullptr;
        h->d_in_flux[d] = nullptr;
        h->d_out_flux[d] = nullptr;
        h->d_src[d] = nullptr;
        h->in_level_beg[d].clear();
        cudaFree(h->d_fcargs[d]);
        h->d_fcargs[d] = nullptr;
    }
    for (auto& b : h->blocks) {
        for (int d = 0; d < 3; ++d) b.fc[d] = FcArgs{};
        cudaFree(b.leaf);
        b.leaf = nullptr;
        b.leaf_cells = -1;
    }
}

template <class T>
int upload_vec(pk_ctx* h, const std::vector<T>& v, T** dev)
{
    *dev = nullptr;
    if (v.empty()) return PK_OK;
    PK_CUDA(h, cudaMalloc(dev, sizeof(T) * v.size()));
    PK_CUDA(h, cudaMemcpy(*dev, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice));
    return PK_OK;
}

// the fine/coarse couplings of a refined domain (build_levels) on the device
int upload_segs(pk_ctx* h, const std::vector<XSeg>& segs, XSegList* out);

// rows of each fine level on the device, start counts relative to the level's first row
static int upload_runs(pk_ctx* h, int maxl, const std::vector<PRun>& pr, const std::vector<long long>& level_beg,
                       PRunDev** d_runs, long long** d_start, std::vector<long long>& beg, std::vector<long long>& cells)
{
    std::vector<PRunDev> runs(pr.size());
    std::vector<long long> start(pr.size());
    beg.assign(level_beg.begin(), level_beg.end());
    cells.assign(maxl + 1, 0);
    for (int L = 1; L <= maxl; ++L) {
        long long acc = 0;
        for (long long r = level_beg[L]; r < level_beg[L + 1]; ++r) {
            const PRun& s = pr[r];
            runs[r] = PRunDev{s.fb, s.cb, s.fx, s.fy, s.fz, s.len, s.cx, s.cy, s.cz, s.px, s.py, s.pz};
            start[r] = acc;
            acc += s.len;
        }
        cells[L] = acc;
    }
    if (int rc = upload_vec(h, runs, d_runs)) return rc;
    return upload_vec(h, start, d_start);
}

int levels_prepare(pk_ctx* h, const std::vector<XSeg>& segs)
{
    const int nl = (int)h->blocks.size();
    std::vector<LBlock> lb(nl);
    double dl0[3] = {0, 0, 0};
    for (int i = 0; i < nl; ++i)
        if (h->blocks[i].level == 0)
            for (int d = 0; d < 3; ++d) dl0[d] = h->blocks[i].dl[d];
    for (int i = 0; i < nl; ++i) {
        const Block& b = h->blocks[i];
        lb[i].level = b.level;
        for (int d = 0; d < 3; ++d) {
            lb[i].n[d] = b.n[d];
            lb[i].g[d] = b.g[d];
            lb[i].off[d] = b.off[d];
            if (h->dom[d] > 1 && b.dl[d] != std::ldexp(dl0[d], -b.level))
                return fail(h, PK_E_ARG, "a block's cell size must be the base cell size / 2**level");
        }
    }
    for (int d = 0; d < 3; ++d)
        if (h->dom[d] > 1 && !h->dom_periodic[d])
            return fail(h, PK_E_UNSUPPORTED, "refined domains are periodic in every direction");
    LevelPlan plan;
    std::string err;
    if (!build_levels(lb, h->dom, plan, err)) return fail(h, PK_E_ARG, err);
    free_levels(h);
    const int NV = h->nplanes;
    if (int rc = upload_runs(h, plan.max_level, plan.runs, plan.run_level_beg, &h->d_runs, &h->d_run_start, h->run_beg,
                             h->run_cells))
        return rc;
    // the partial refreshes of the batched stage path, one per swept direction
    const int rmax = std::max(h->pro_u.r, h->pro_b.r);
    for (int d = 0; d < 3; ++d) {
        if (h->dom[d] <= 1) continue;
        PartialRefresh pr;
        build_partial_refresh(lb, plan, segs, d, rmax, pr);
        pk_ctx::Partial& q = h->part[d];
        if (int rc = upload_segs(h, pr.segs, &q.segs)) return rc;
        if (int rc = upload_runs(h, plan.max_level, pr.runs, pr.run_level_beg, &q.runs, &q.run_start, q.run_beg,
                                 q.run_cells))
            return rc;
        q.ok = true;
    }
    // per direction: the blocks' slot tables, then in faces, then flux sources
    for (int d = 0; d < 3; ++d) {
        const FcDir& F = plan.fc[d];
        h->in_level_beg[d] = F.in_level_beg;
        std::vector<int> ints;
        std::vector<long long> in_off(nl, -1), out_off(nl, -1);
        for (int i = 0; i < nl; ++i) {
            if (!F.in_slot[i].empty()) {
                in_off[i] = (long long)ints.size();
                ints.insert(ints.end(), F.in_slot[i].begin(), F.in_slot[i].end());
            }
            if (!F.out_slot[i].empty()) {
                out_off[i] = (long long)ints.size();
                ints.insert(ints.end(), F.out_slot[i].begin(), F.out_slot[i].end());
            }
        }
        const long long face_off = (long long)ints.size();
        ints.insert(ints.end(), F.in_face.begin(), F.in_face.end());
        const long long src_off = (long long)ints.size();
        ints.insert(ints.end(), F.src.begin(), F.src.end());
        if (int rc = upload_vec(h, ints, &h->d_fc_int[d])) return rc;
        const size_t nin = F.in_face.size();
        if (nin) PK_CUDA(h, cudaMalloc(&h->d_in_flux[d], sizeof(double) * NV * nin));
        if (F.n_out) PK_CUDA(h, cudaMalloc(&h->d_out_flux[d], sizeof(double) * NV * F.n_out));
        h->d_src[d] = nin ? h->d_fc_int[d] + src_off : nullptr;
        std::vector<FcArgs> tab(nl);
        for (int i = 0; i < nl; ++i) {
            FcArgs& f = h->blocks[i].fc[d];
            f.in_slot = in_off[i] >= 0 ? h->d_fc_int[d] + in_off[i] : nullptr;
            f.in_face = nin ? h->d_fc_int[d] + face_off : nullptr;
            f.in_flux = h->d_in_flux[d];
            f.out_slot = out_off[i] >= 0 ? h->d_fc_int[d] + out_off[i] : nullptr;
            f.out_flux = h->d_out_flux[d];
            tab[i] = f;
        }
        if (nin || F.n_out)
            if (int rc = upload_vec(h, tab, &h->d_fcargs[d])) return rc;
    }
    for (int i = 0; i < nl; ++i) {
        Block& b = h->blocks[i];
        b.leaf_cells = plan.leaf_cells[i];
        if (!plan.leaf[i].empty())
            if (int rc = upload_vec(h, plan.leaf[i], &b.leaf)) return rc;
    }
    // restriction targets, start counts relative to each fine level's first box
    std::vector<RBoxDev> rb(plan.rboxes.size());
    std::vector<long long> rstart(plan.rboxes.size());
    h->rbox_beg.assign(plan.rbox_level_beg.begin(), plan.rbox_level_beg.end());
    h->rbox_cells.assign(plan.max_level + 1, 0);
    for (int L = 1; L <= plan.max_level; ++L) {
        long long acc = 0;
        for (int r = plan.rbox_level_beg[L]; r < plan.rbox_level_beg[L + 1]; ++r) {
            const RBox& s = plan.rboxes[r];
            RBoxDev& d = rb[r];
            d.fb = s.fb;
            d.cb = s.cb;
            long long cells = 1;
            for (int k = 0; k < 3; ++k) {
                d.lo[k] = s.lo[k];
                d.hi[k] = s.hi[k];
                d.flo[k] = s.flo[k];
                cells *= s.hi[k] - s.lo[k];
            }
            rstart[r] = acc;
            acc += cells;
        }
        h->rbox_cells[L] = acc;
    }
    if (int rc = upload_vec(h, rb, &h->d_rbox)) return rc;
    if (int rc = upload_vec(h, rstart, &h->d_rbox_start)) return rc;
    h->eff_dim = plan.eff_dim;
    h->fc_scale = 1.0 / std::ldexp(1.0, plan.eff_dim - 1);
    h->max_level = plan.max_level;
    h->batch_dirty = true;
    return PK_OK;
}

// The directional stencil of a prolongation order (grid_container_prolong.F90:
// 223-287 select case (ord_prolong)): P_3..P3 and the stencil range; every
// coefficient is a dyadic fraction, exact in binary64.  false: unknown order.
bool prolong_coef(int order, ProlongCoef* k)
{
    double P[7] = {0, 0, 0, 0, 0, 0, 0};      // P_3, P_2, P_1, P0, P1, P2, P3
    int r;
    switch (order) {
    case -6: P[0] = -231.0 / 65536; P[1] = 2002.0 / 65536; P[2] = -9009.0 / 65536; P[3] = 60060.0 / 65536;
             P[4] = 15015.0 / 65536; P[5] = -2574.0 / 65536; P[6] = 273.0 / 65536; r = 3; break;
    case -5: P[1] = 77.0 / 8192; P[2] = -693.0 / 8192; P[3] = 6930.0 / 8192; P[4] = 2310.0 / 8192;
             P[5] = -495.0 / 8192; P[6] = 63.0 / 8192; r = 3; break;
    case -4: P[1] = 35.0 / 2048; P[2] = -252.0 / 2048; P[3] = 1890.0 / 2048; P[4] = 420.0 / 2048;
             P[5] = -45.0 / 2048; r = 2; break;
    case -3: P[2] = -7.0 / 128; P[3] = 105.0 / 128; P[4] = 35.0 / 128; P[5] = -5.0 / 128; r = 2; break;
    case -2: P[2] = -3.0 / 32; P[3] = 30.0 / 32; P[4] = 5.0 / 32; r = 1; break;
    case 1: P[3] = 3.0 / 4; P[4] = 1.0 / 4; r = 1; break;                      // O_LIN
    case 0: P[3] = 1.0; r = 0; break;                                         // O_INJ
    case 2: P[2] = -1.0 / 8; P[3] = 1.0; P[4] = 1.0 / 8; r = 1; break;
    case 3: P[2] = -5.0 / 64; P[3] = 55.0 / 64; P[4] = 17.0 / 64; P[5] = -3.0 / 64; r = 2; break;
    case 4: P[1] = 3.0 / 128; P[2] = -11.0 / 64; P[3] = 1.0; P[4] = 11.0 / 64; P[5] = -3.0 / 128; r = 2; break;
    case 5: P[1] = 7.0 / 512; P[2] = -63.0 / 512; P[3] = 462.0 / 512; P[4] = 138.0 / 512; P[5] = -37.0 / 512;
            P[6] = 5.0 / 512; r = 3; break;
    case 6: P[0] = -5.0 / 1024; P[1] = 44.0 / 1024; P[2] = -201.0 / 1024; P[3] = 1.0; P[4] = 201.0 / 1024;
            P[5] = -44.0 / 1024; P[6] = 5.0 / 1024; r = 3; break;
    default: return false;
    }
    for (int i = 0; i < 7; ++i) k->p[i] = P[i];
    k->r = r;
    return true;
}

// prolong_bnd_from_coarser of every refined level, coarsest first
int prolong_guards(pk_ctx* h, int need = -1, int parity = -1)
{
    const bool part = need >= 0 && h->part[need].ok;
    const std::vector<long long>& beg = part ? h->part[need].run_beg : h->run_beg;
    const std::vector<long long>& cnt = part ? h->part[need].run_cells : h->run_cells;
    const PRunDev* rows = part ? h->part[need].runs : h->d_runs;
    const long long* rstart = part ? h->part[need].run_start : h->d_run_start;
    for (int L = 1; L <= h->max_level; ++L) {
        const long long cells = cnt[L];
        if (!cells) continue;
        const long long r0 = beg[L];
        const int nr = (int)(beg[L + 1] - r0);
        k_prolong<<<grid1d(cells, 256), 256, 0, h->stream>>>(rows + r0, rstart + r0, nr, cells,
                                                             h->d_xptr[parity < 0 ? h->cur : parity], h->nvf,
                                                             h->cfg.magnetic ? 4 : 0,
                                                             h->dom[0] > 1, h->dom[1] > 1, h->dom[2] > 1, h->pro_u,
                                                             h->pro_b, h->pro_b);
        PK_CUDA(h, cudaGetLastError());
        h->launches += 1;
    }
    return PK_OK;
}

int exchange_prepare(pk_ctx* h)
{
    if (!h->connected) return PK_OK;
    const int nl = (int)h->blocks.size();
    int maxl = 0;
    for (auto& b : h->blocks) maxl = std::max(maxl, b.level);
    if (h->x_dirty && maxl > 0) {
        // one exchange plan per level, on that level's grid
        if (!h->remote.empty()) return fail(h, PK_E_UNSUPPORTED, "refined domains run on one rank");
        std::vector<XSeg> all;
        for (int L = 0; L <= maxl; ++L) {
            std::vector<int> ids;
            std::vector<XBlock> xb;
            for (int i = 0; i < nl; ++i) {
                const Block& b = h->blocks[i];
                if (!b.placed) return fail(h, PK_E_STATE, "every block of a connected domain must be placed (pk_block_place)");
                if (b.level != L) continue;
                XBlock x;
                for (int d = 0; d < 3; ++d) {
                    x.n[d] = b.n[d];
                    x.g[d] = b.g[d];
                    x.off[d] = b.off[d];
                }
                ids.push_back(i);
                xb.push_back(x);
            }
            long long dom[3];
            for (int d = 0; d < 3; ++d) dom[d] = h->dom[d] > 1 ? h->dom[d] << L : 1;
            std::vector<XSeg> segs;
            std::string err;
            if (!build_exchange(xb, dom, h->dom_periodic, segs, err)) return fail(h, PK_E_ARG, err);
            for (XSeg s : segs) {
                s.dst = ids[s.dst];
                s.src = ids[s.src];
                all.push_back(s);
            }
        }
        if (int rc = levels_prepare(h, all)) return rc;
        PK_CUDA(h, cudaStreamSynchronize(h->stream));
        free_segs(h);
        if (int rc = upload_segs(h, all, &h->xlocal)) return rc;
        h->x_dirty = false;
    }
    if (h->x_dirty && h->max_level > 0) {              // no longer refined
        free_levels(h);
        h->max_level = 0;
        h->batch_dirty = true;
    }
    if (h->x_dirty) {
        // this rank's blocks first, then the other ranks'
        std::vector<XBlock> xb(nl + h->remote.size());
        std::vector<int> owner(xb.size(), -1);
        for (int i = 0; i < nl; ++i) {
            const Block& b = h->blocks[i];
            if (!b.placed) return fail(h, PK_E_STATE, "every block of a connected domain must be placed (pk_block_place)");
            for (int d = 0; d < 3; ++d) {
                xb[i].n[d] = b.n[d];
                xb[i].g[d] = b.g[d];
                xb[i].off[d] = b.off[d];
            }
        }
        for (size_t r = 0; r < h->remote.size(); ++r) {
            const RemoteBlock& rb = h->remote[r];
            XBlock& x = xb[nl + r];
            for (int d = 0; d < 3; ++d) {
                x.n[d] = rb.n[d];
                x.g[d] = rb.n[d] > 1 ? h->cfg.nb : 0;
                x.off[d] = rb.off[d];
            }
            owner[nl + r] = rb.owner;
        }
        std::vector<XSeg> segs, local;
        std::vector<XPeer> peers;
        std::string err;
        if (!build_exchange(xb, h->dom, h->dom_periodic, segs, err)) return fail(h, PK_E_ARG, err);
        split_by_owner(xb, owner, nl, segs, local, peers);
        PK_CUDA(h, cudaStreamSynchronize(h->stream));
        free_segs(h);
        if (int rc = upload_segs(h, local, &h->xlocal)) return rc;
        for (int d = 0; d < 3; ++d)
            if (int rc = upload_segs(h, face_segs(xb, local, d), &h->xlocal_dir[d])) return rc;
        for (const XPeer& p : peers) {
            XPeerDev d;
            d.rank = p.rank;
            h->xpeers.push_back(d);
            XPeerDev& q = h->xpeers.back();
            if (int rc = upload_segs(h, p.send, &q.send)) return rc;
            if (int rc = upload_segs(h, p.recv, &q.recv)) return rc;
            for (int k = 0; k < 3; ++k) {   // canonical order kept: both sides filter their lists alike
                if (int rc = upload_segs(h, face_segs(xb, p.send, k), &q.send_dir[k])) return rc;
                if (int rc = upload_segs(h, face_segs(xb, p.recv, k), &q.recv_dir[k])) return rc;
            }
        }
        h->x_dir = true;
        h->x_dirty = false;
    }
    if (h->x_ptrs_dirty) {
        if (int rc = ensure_pingpong(h)) return rc;
        std::vector<XPtr> ptr(nl);
        PK_CUDA(h, cudaStreamSynchronize(h->stream));
        for (int p = 0; p < 2; ++p) {
            for (int i = 0; i < nl; ++i) {
                const Block& b = h->blocks[i];
                ptr[i].u = b.buf[p];
                ptr[i].plane = b.plane;
                for (int d = 0; d < 3; ++d) ptr[i].ext[d] = b.ext[d];
            }
            cudaFree(h->d_xptr[p]);
            h->d_xptr[p] = nullptr;
            PK_CUDA(h, cudaMalloc(&h->d_xptr[p], sizeof(XPtr) * (nl > 0 ? nl : 1)));
            PK_CUDA(h, cudaMemcpy(h->d_xptr[p], ptr.data(), sizeof(XPtr) * nl, cudaMemcpyHostToDevice));
        }
        h->x_ptrs_dirty = false;
    }
    return PK_OK;
}

// launch the exchange between this rank's blocks on the current state, then
// let the host move the other ranks' halo.  dir >= 0: only the face boxes
// along dir, all a fused sweep along dir reads (called right before it);
// -1: every guard cell
// need >= 0: only the guard cells the interior-trimmed stage kernel reads
// when it next sweeps direction need (refined domains; every other guard cell
// may stay stale until a full refresh)
int exchange_guards(pk_ctx* h, int dir = -1, int need = -1)
{
    if (!h->connected) return PK_OK;
    if (int rc = exchange_prepare(h)) return rc;
    if (need >= 0 && !(h->max_level > 0 && h->part[need].ok)) need = -1;
    // before a fused sweep along dir only the face boxes along dir are read
    const XSegList& xs = need >= 0 ? h->part[need].segs
                                   : ((dir >= 0 && h->x_dir && h->max_level == 0) ? h->xlocal_dir[dir] : h->xlocal);
    if (xs.total > 0) {
        const int nblk = (int)(xs.n < grid_cap() ? xs.n : grid_cap());   // CTAs take whole segments
        k_exchange<<<nblk, 256, 0, h->stream>>>(xs.dev, xs.n, xs.total, h->d_xptr[h->cur], h->nplanes);
        PK_CUDA(h, cudaGetLastError());
        h->launches += 1;
    }
    if (h->halo_cb && !h->xpeers.empty()) h->halo_cb(h->comm_ctx, dir);
    if (h->max_level > 0) return prolong_guards(h, need);
    return PK_OK;
}

// Guard cells of a block whose sweeps left them stale: its own boundary rules,
// and for a connected domain every block's exchange.
int refresh_guards(pk_ctx* h, Block& b)
{
    if (!h->connected) return fill_guards_block(h, b);
    for (auto& c : h->blocks)
        if (int rc = fill_guards_block(h, c)) return rc;
    return exchange_guards(h);
}

// A connected domain sweeps with the fused kernels when the blocks tile a
// domain periodic in every swept direction: the exchange before each sweep
// then fills every guard cell, and the kernels read their 4-cell halo from
// the guards -- the same values a periodic single block reads by wrapping.
bool connected_fused_ok(pk_ctx* h)
{
    long long cells = 0;
    for (auto& b : h->blocks) {
        if (!b.placed) return false;
        cells += (long long)b.n[0] * b.n[1] * b.n[2];
    }
    for (auto& r : h->remote) cells += (long long)r.n[0] * r.n[1] * r.n[2];
    for (int d = 0; d < 3; ++d)
        if (h->dom[d] > 1 && !h->dom_periodic[d]) return false;
    return cells == h->dom[0] * h->dom[1] * h->dom[2];
}

bool fused_ok(pk_ctx* h)
{
    if (h->cfg.integration_order != 2) return false;
    for (auto& b : h->blocks)
        if (b.level > 0) return false;                 // refined domains sweep stage by stage
    if (h->connected) return connected_fused_ok(h);
    for (auto& b : h->blocks)
        for (int d = 0; d < 3; ++d)
            if (b.n[d] > 1 && (b.bnd[d][0] != PK_BND_PER || b.bnd[d][1] != PK_BND_PER)) return false;
    return true;
}

int ensure_pingpong(pk_ctx* h)
{
    for (auto& b : h->blocks)
        if (!b.buf[1 - h->cur]) {
            double* p = nullptr;
            PK_CUDA(h, cudaMalloc(&p, sizeof(double) * h->nplanes * b.plane));
            PK_CUDA(h, cudaMemsetAsync(p, 0, sizeof(double) * h->nplanes * b.plane, h->stream));
            b.buf[1 - h->cur] = p;
            h->batch_dirty = true;
            h->x_ptrs_dirty = true;
        }
    return PK_OK;
}

// block tables (both parities) and per-direction work lists of the batched sweep
// The one-launch work list of a refined stage along dir (k_stage_refined):
// first every stage item of a block without replaced fluxes, finest level
// first; then per coarse level, finest first, the restriction chunks of its in
// slots (each waits for all stage items of the level above) and the stage
// items of its blocks with replaced fluxes (each waits for all of those
// chunks).  Every item comes after all items it waits for.
int build_refined_list(pk_ctx* h, int dir, const std::vector<std::vector<StageItem>>& items, int maxl)
{
    constexpr int CHUNK = 64;                         // in slots per restriction chunk
    const int nlev = maxl + 1;
    auto dependent = [&](int blk) { return h->blocks[blk].fc[dir].in_slot != nullptr; };
    auto stage_item = [&](const StageItem& w, int level, int wait, int count) {
        RefItem r{};
        r.kind = 0;
        r.block = w.block;
        r.i1_0 = w.i1_0;
        r.P = w.P;
        r.level = level;
        r.wait = wait;
        r.wait_count = count;
        r.fence = h->blocks[w.block].fc[dir].out_slot != nullptr;
        return r;
    };
    std::vector<RefItem> ri;
    for (int L = maxl; L >= 0; --L)
        for (const StageItem& w : items[L])
            if (!dependent(w.block)) ri.push_back(stage_item(w, L, -1, 0));
    for (int L = maxl; L >= 1; --L) {
        const int cl = L - 1;
        int nchunk = 0;
        if (h->d_src[dir] && (int)h->in_level_beg[dir].size() > L) {
            const int beg = h->in_level_beg[dir][cl], end = h->in_level_beg[dir][L];
            for (int s0 = beg; s0 < end; s0 += CHUNK) {
                RefItem r{};
                r.kind = 1;
                r.level = cl;
                r.beg = s0;
                r.end = std::min(s0 + CHUNK, end);
                r.wait = 1 + L;                       // every stage item of level L done
                r.wait_count = (int)items[L].size();
                r.fence = 1;
                ri.push_back(r);
                ++nchunk;
            }
        }
        for (const StageItem& w : items[cl])
            if (dependent(w.block)) ri.push_back(stage_item(w, cl, nchunk ? 1 + nlev + cl : -1, nchunk));
    }
    size_t smem = 0;
    for (const StageList& sl : h->sbatch[dir]) smem = std::max(smem, sl.smem);
    cudaFree(h->rdev[dir]);
    h->rdev[dir] = nullptr;
    h->rn[dir] = (int)ri.size();
    h->rsmem[dir] = smem;
    if (!ri.empty()) {
        PK_CUDA(h, cudaMalloc(&h->rdev[dir], sizeof(RefItem) * ri.size()));
        PK_CUDA(h, cudaMemcpyAsync(h->rdev[dir], ri.data(), sizeof(RefItem) * ri.size(), cudaMemcpyHostToDevice,
                                   h->stream));
        PK_CUDA(h, cudaStreamSynchronize(h->stream));
    }
    if (h->rcount_n < 1 + 2 * nlev) {
        cudaFree(h->d_rcount);
    cudaFree(h->d_eglm);
        h->d_rcount = nullptr;
        h->rcount_n = 1 + 2 * nlev;
        PK_CUDA(h, cudaMalloc(&h->d_rcount, sizeof(unsigned) * h->rcount_n));
    }
    return PK_OK;
}

int build_batch(pk_ctx* h)
{
    if (int rc = ensure_pingpong(h)) return rc;
    if (!h->batch_dirty) return PK_OK;
    const int nb = (int)h->blocks.size();
    if (!fused_ok(h))                                  // the stage path keeps cg%w(uh) per block
        for (auto& b : h->blocks)
            if (!b.uh) PK_CUDA(h, cudaMalloc(&b.uh, sizeof(double) * h->nplanes * b.plane));
    std::vector<BlockDesc> desc(nb);
    for (int p = 0; p < 2; ++p) {
        for (int i = 0; i < nb; ++i) {
            const Block& b = h->blocks[i];
            BlockDesc& d = desc[i];
            d.in = b.buf[p];
            d.out = b.buf[1 - p];
            d.plane = b.plane;
            for (int k = 0; k < 3; ++k) {
                d.ext[k] = b.ext[k];
                d.g[k] = b.g[k];
                d.n[k] = b.n[k];
                d.dl[k] = b.dl[k];
            }
            d.wrap = h->connected ? 0 : 1;
            d.leaf = b.leaf;
            d.uh = b.uh;
        }
        cudaFree(h->d_desc[p]);
        h->d_desc[p] = nullptr;
        PK_CUDA(h, cudaMalloc(&h->d_desc[p], sizeof(BlockDesc) * (nb > 0 ? nb : 1)));
        PK_CUDA(h, cudaMemcpyAsync(h->d_desc[p], desc.data(), sizeof(BlockDesc) * nb, cudaMemcpyHostToDevice, h->stream));
        PK_CUDA(h, cudaStreamSynchronize(h->stream));   // desc is reused for the other parity
    }
    const int threads = VAR_T[h->pp.weno3 ? W3_VARIANT : h->batch_variant];
    for (int dir = 0; dir < 3; ++dir) {
        BatchList& bl = h->batch[dir];
        bl.host.clear();
        const int o1 = ORTHO1[dir], o2 = ORTHO2[dir];
        for (int i = 0; i < nb; ++i) {
            const Block& b = h->blocks[i];
            if (b.n[dir] <= 1) continue;
            // a periodic pencil that fits the CTA is swept whole, without halo
            const int circ = (!h->connected && b.n[dir] <= threads && h->batch_circ) ? 1 : 0;
            const int L = circ ? b.n[dir] : (b.n[dir] < h->batch_L ? b.n[dir] : h->batch_L);
            const int T = circ ? L : L + 8;
            if (T > threads) return fail(h, PK_E_ARG, "batched tile longer than the CTA");
            int P = threads / T;
            if (P > b.n[o1]) P = b.n[o1];
            for (int i2 = 0; i2 < b.n[o2]; ++i2)
                for (int c0 = 0; c0 < b.n[dir]; c0 += L)
                    for (int i1 = 0; i1 < b.n[o1]; i1 += P) bl.host.push_back(WorkItem{i, i1, c0, i2, P, L, circ});
        }
        cudaFree(bl.dev);
        bl.dev = nullptr;
        bl.n = (int)bl.host.size();
        if (bl.n) {
            PK_CUDA(h, cudaMalloc(&bl.dev, sizeof(WorkItem) * bl.n));
            PK_CUDA(h, cudaMemcpyAsync(bl.dev, bl.host.data(), sizeof(WorkItem) * bl.n, cudaMemcpyHostToDevice, h->stream));
        }
    }
    // the batched stage: per direction and level, items of P pencils
    const int sv = h->pp.weno3 ? 0 : h->stage_variant;
    int maxl = 0;
    bool fits = true;
    for (auto& b : h->blocks) {
        maxl = std::max(maxl, b.level);
        for (int d = 0; d < 3; ++d) fits = fits && (b.n[d] <= 1 || (b.n[d] + 4 <= SV_T[sv] && b.g[d] >= 3));
    }
    h->stage_batched = fits && nb > 1;
    std::vector<std::vector<StageItem>> items;
    for (int dir = 0; dir < 3; ++dir) {
        for (StageList& s : h->sbatch[dir]) cudaFree(s.dev);
        h->sbatch[dir].assign(maxl + 1, StageList());
        cudaFree(h->rdev[dir]);
        h->rdev[dir] = nullptr;
        h->rn[dir] = 0;
        if (!h->stage_batched) continue;
        items.assign(maxl + 1, {});
        const int o1 = ORTHO1[dir], o2 = ORTHO2[dir];
        for (int i = 0; i < nb; ++i) {
            const Block& b = h->blocks[i];
            if (b.n[dir] <= 1) continue;
            const int T = b.n[dir] + 4;                 // the trimmed tile of k_stage_batched
            const int face = b.n[o1] * b.n[o2];         // pencils, taken in i1-fastest order across i2 rows
            int P = SV_T[sv] / T;
            if (P > face) P = face;
            StageList& sl = h->sbatch[dir][b.level];
            sl.smem = std::max(sl.smem, (size_t)3 * h->nplanes * P * T * sizeof(double));
            for (int q = 0; q < face; q += P) items[b.level].push_back(StageItem{i, q, 0, P});
        }
        for (int L = 0; L <= maxl; ++L) {
            StageList& sl = h->sbatch[dir][L];
            sl.n = (int)items[L].size();
            if (!sl.n) continue;
            PK_CUDA(h, cudaMalloc(&sl.dev, sizeof(StageItem) * sl.n));
            PK_CUDA(h, cudaMemcpyAsync(sl.dev, items[L].data(), sizeof(StageItem) * sl.n, cudaMemcpyHostToDevice,
                                       h->stream));
            PK_CUDA(h, cudaStreamSynchronize(h->stream));
        }
        if (maxl > 0)
            if (int rc = build_refined_list(h, dir, items, maxl)) return rc;
    }
    PK_CUDA(h, cudaStreamSynchronize(h->stream));   // host vectors of the tables may change after return
    h->batch_dirty = false;
    return PK_OK;
}

void invalidate_graph(pk_ctx* h)
{
    if (h->graph_exec) cudaGraphExecDestroy(h->graph_exec);
    if (h->graph) cudaGraphDestroy(h->graph);
    h->graph_exec = nullptr;
    h->graph = nullptr;
}

int put_step_params(pk_ctx* h, double dt, double ch, double fac)
{
    PK_CUDA(h, cudaStreamSynchronize(h->stream));   // the previous copy out of h_step has completed
    for (int i = 0; i < h->ninst; ++i) {
        h->h_step[i].dt = dt;
        h->h_step[i].ch = ch;
        h->h_step[i].psi_fac = fac;
    }
    PK_CUDA(h, cudaMemcpyAsync(h->d_step, h->h_step, sizeof(StepParams) * h->ninst, cudaMemcpyHostToDevice, h->stream));
    return PK_OK;
}

// one set of step scalars per instance
int put_step_array(pk_ctx* h, const StepRec* r)
{
    PK_CUDA(h, cudaStreamSynchronize(h->stream));
    for (int i = 0; i < h->ninst; ++i) {
        h->h_step[i].dt = r[i].dt;
        h->h_step[i].ch = r[i].ch;
        h->h_step[i].psi_fac = r[i].fac;
    }
    PK_CUDA(h, cudaMemcpyAsync(h->d_step, h->h_step, sizeof(StepParams) * h->ninst, cudaMemcpyHostToDevice, h->stream));
    return PK_OK;
}

// glmdamping with the step's factor read from d_step (graph-safe)
int glm_scale_dev(pk_ctx* h)
{
    if (h->blocks.size() > 1) {
        if (int rc = build_batch(h)) return rc;
        long long mp = 0;
        for (auto& b : h->blocks) mp = std::max(mp, b.plane);
        long long gx = (mp + 255) / 256;
        if (gx > 64) gx = 64;
        k_scale_blocks<<<dim3((unsigned)gx, (unsigned)h->blocks.size()), 256, 0, h->stream>>>(h->d_desc[h->cur], h->ib + 3,
                                                                                         h->d_step);
        PK_CUDA(h, cudaGetLastError());
        h->launches += 1;
        return PK_OK;
    }
    for (auto& b : h->blocks) {
        k_scale_dev<<<grid1d(b.plane, 256), 256, 0, h->stream>>>(state(h, b) + (long long)(h->ib + 3) * b.plane, b.plane,
                                                                 h->d_step);
        PK_CUDA(h, cudaGetLastError());
        h->launches += 1;
    }
    return PK_OK;
}

int glm_scale(pk_ctx* h, double fac)
{
    for (auto& b : h->blocks) {
        k_scale<<<grid1d(b.plane, 256), 256, 0, h->stream>>>(state(h, b) + (long long)(h->ib + 3) * b.plane, b.plane, fac);
        PK_CUDA(h, cudaGetLastError());
        h->launches += 1;
    }
    return PK_OK;
}

// sweep(cdim) of all blocks; the step scalars are already in d_step.
// apply_fac: the psi damping of glmdamping is folded into this sweep.
// next_dir: the direction the following sweep of the same step takes (-1:
// none, so the last guard refresh is complete)
int sweep_impl(pk_ctx* h, int dir, double dt, double ch, int apply_fac, double fac, int next_dir = -1)
{
    if (h->blocks.empty()) return fail(h, PK_E_STATE, "no block registered");
    const PhysOps* ops = ops_of(h);
    if (fused_ok(h)) {
        if (int rc = ensure_pingpong(h)) return rc;
        if (int rc = exchange_guards(h, dir)) return rc;   // connected domains: halos come from the guards
        const FastOps* fo = h->arith == PK_ARITH_FMA ? fast_ops_of(h) : nullptr;
        if ((h->batched && h->ninst < 2) || h->blocks.size() > 1) {
            if (int rc = build_batch(h)) return rc;
            if (int rc = fo ? fo->batched(h, dir, apply_fac, h->d_counter + dir)
                            : ops->batched(h, dir, apply_fac, h->d_counter + dir))
                return rc;
            for (auto& b : h->blocks) b.guards_stale = true;
        } else {
            for (auto& b : h->blocks)
                if (b.n[dir] > 1)
                    if (int rc = fo ? fo->fused(h, b, dir, apply_fac) : ops->fused(h, b, dir, apply_fac)) return rc;
        }
        h->cur ^= 1;
        return PK_OK;
    }
    const int nst = h->cfg.integration_order == 1 ? 1 : 2;
    if (int rc = exchange_prepare(h)) return rc;       // a refined domain's couplings
    if (h->blocks.size() > 1)
        if (int rc = build_batch(h)) return rc;
    const bool one_launch = h->stage_batched && h->max_level > 0 && h->refined_one_launch && h->rn[dir] > 0;
    for (int s = 1; s <= nst; ++s) {
        const double rk = (h->cfg.integration_order == 1) ? 1.0 : (s == 1 ? 0.5 : 1.0);
        // finest level first: its boundary fluxes replace the coarser level's (sweeps.F90:218-262)
        if (one_launch)
            if (int rc = ops->stage_refined(h, dir, s == 1, rk)) return rc;
        for (int L = one_launch ? -1 : h->max_level; L >= 0; --L) {
            if (h->stage_batched) {
                if (int rc = ops->stage_batched(h, dir, L, s == 1, rk)) return rc;
            } else {
                for (auto& b : h->blocks) {
                    if (b.n[dir] <= 1 || b.level != L) continue;
                    if (!b.uh) PK_CUDA(h, cudaMalloc(&b.uh, sizeof(double) * h->nplanes * b.plane));
                    if (stage_chunked(b, dir))
                        if (int rc = ensure_pingpong(h)) return rc;
                    if (int rc = ops->stage(h, b, dir, s == 1, rk)) return rc;
                }
            }
            if (L > 0 && h->d_src[dir]) {
                const int beg = h->in_level_beg[dir][L - 1], end = h->in_level_beg[dir][L];
                if (end > beg) {
                    const long long n = (long long)(end - beg) * h->nplanes;
                    k_restrict_flux<<<grid1d(n, 256), 256, 0, h->stream>>>(h->d_src[dir], beg, end, h->nplanes,
                                                                           h->d_out_flux[dir], h->d_in_flux[dir],
                                                                           h->fc_scale);
                    PK_CUDA(h, cudaGetLastError());
                    h->launches += 1;
                }
            }
        }
        if (h->max_level == 0)                        // refined domains overwrite every guard cell below
            for (auto& b : h->blocks)
                if (int rc = fill_guards_block(h, b)) return rc;
        // the batched stage reads two guard layers along the next stage's direction only
        const int need = !h->stage_batched ? -1 : (s < nst ? dir : next_dir);
        if (int rc = exchange_guards(h, -1, need)) return rc;   // every guard cell (the next sweep's too)
    }
    if (h->cfg.magnetic && apply_fac) return glm_scale_dev(h);
    return PK_OK;
}

double min_dl(pk_ctx* h, int* eff)
{
    double m = DBL_MAX;
    int e = 0;
    for (auto& b : h->blocks)
        for (int d = 0; d < 3; ++d)
            if (b.n[d] > 1) {
                m = (b.dl[d] < m) ? b.dl[d] : m;
                e = 1;
            }
    if (eff) *eff = e;
    return m;
}

void step_dirs(pk_ctx* h, int* dirs, int* nd)
{
    *nd = 0;
    for (int d = 0; d < 3; ++d) {
        bool has = false;
        for (auto& b : h->blocks) has = has || b.n[d] > 1;
        if (has && !h->cfg.skip_sweep[d]) dirs[(*nd)++] = d;
    }
}

// the launches of fluid_update_full after the step scalars are on the device
// E-GLM scratch for the largest block (outside any graph capture)
int eglm_alloc(pk_ctx* h)
{
    if (!(h->cfg.use_eglm && h->cfg.magnetic)) return PK_OK;
    long long mp = 0;
    for (auto& b : h->blocks) mp = std::max(mp, b.plane);
    if (mp <= h->eglm_plane) return PK_OK;
    cudaFree(h->d_eglm);
    h->d_eglm = nullptr;
    h->eglm_plane = 0;
    if (cudaMalloc(&h->d_eglm, sizeof(double) * 4 * mp) != cudaSuccess)
        return fail(h, PK_E_NOMEM, "cudaMalloc for the E-GLM scratch failed");
    h->eglm_plane = mp;
    return PK_OK;
}

// every guard cell of every block from the current state (the reference's
// boundary updates at the end of each sweep and of eglm)
int refresh_all(pk_ctx* h)
{
    if (h->connected) return refresh_guards(h, h->blocks[0]);
    for (auto& b : h->blocks)
        if (int rc = fill_guards_block(h, b)) return rc;
    return PK_OK;
}

// eglm (hdc.F90:355-457) on every block: guards refreshed, divB and grad(psi)
// of all interior cells, the sources, the boundary update; dt from d_step
int eglm_dev(pk_ctx* h)
{
    if (h->max_level > 0) return fail(h, PK_E_UNSUPPORTED, "use_eglm on refined domains");
    if (h->ninst > 1) return fail(h, PK_E_UNSUPPORTED, "use_eglm with stacked instances");
    if (int rc = eglm_alloc(h)) return rc;
    if (int rc = refresh_all(h)) return rc;
    int idn = -1, off = 0;
    for (int f = 0; f < h->cfg.nfluids; ++f) {
        if (h->cfg.fluid_kind[f] == PK_FLUID_ION && idn < 0) idn = off;
        off += h->cfg.fluid_kind[f] == PK_FLUID_DST ? 4 : 5;
    }
    if (idn >= 0) {
        for (auto& b : h->blocks) {
            EglmArgs a;
            for (int d = 0; d < 3; ++d) {
                a.n[d] = b.n[d];
                a.g[d] = b.g[d];
                a.ext[d] = b.ext[d];
                a.D[d] = b.n[d] > 1 ? 1 : 0;
                a.dl[d] = b.dl[d];
            }
            a.plane = b.plane;
            a.ib = h->ib;
            a.idn = idn;
            const long long cells = (long long)b.n[0] * b.n[1] * b.n[2];
            k_eglm_grad<<<grid1d(cells, 256), 256, 0, h->stream>>>(state(h, b), h->d_eglm, a);
            PK_CUDA(h, cudaGetLastError());
            k_eglm_apply<<<grid1d(cells, 256), 256, 0, h->stream>>>(state(h, b), h->d_eglm, a, h->d_step);
            PK_CUDA(h, cudaGetLastError());
            h->launches += 2;
        }
    }
    return refresh_all(h);
}

int step_sweeps(pk_ctx* h, double dt, double ch, double fac)
{
    int dirs[3], nd;
    step_dirs(h, dirs, &nd);
    // use_eglm: eglm runs between the triple's last sweep and glmdamping
    // (fluidupdate.F90:229-230), so the damping is not fused into that sweep
    const bool eglm = h->cfg.use_eglm && h->cfg.magnetic;
    for (int half = 0; half < 2; ++half) {
        for (int s = 0; s < nd; ++s) {
            const int d = half == 0 ? dirs[s] : dirs[nd - 1 - s];
            const int last = h->cfg.magnetic && s == nd - 1 && !eglm;
            int next = -1;                                // the sweep after this one in the same step
            if (half == 0) next = s + 1 < nd ? dirs[s + 1] : dirs[nd - 1];
            else if (s + 1 < nd) next = dirs[nd - 2 - s];
            if (int rc = sweep_impl(h, d, dt, ch, last, fac, next)) return rc;
        }
        if (eglm) {
            if (int rc = eglm_dev(h)) return rc;
            if (nd > 0)
                if (int rc = glm_scale_dev(h)) return rc;
        }
        if (h->cfg.magnetic && nd == 0)
            if (int rc = glm_scale(h, fac)) return rc;
    }
    return PK_OK;
}

// update_chspeed and the glmdamping factor for dt (hdc.F90:112-119, 310-330)
// update_chspeed with ch_grid = .false. (hdc.F90:118-131,138): the maximum of
// point_chspeed over the leaf cells of every block, then over ranks
int gas_chspeed(pk_ctx* h, double* ch)
{
    if (h->ninst > 1) return fail(h, PK_E_UNSUPPORTED, "ch_grid = 0 with stacked instances");
    if (int rc = exchange_prepare(h)) return rc;      // a refined domain's leaf masks
    if (int rc = build_batch(h)) return rc;           // the block table of the current parity
    if (!h->d_ch) PK_CUDA(h, cudaMalloc(&h->d_ch, sizeof(unsigned long long)));
    ChArgs a;
    a.kind = h->cfg.fluid_kind[0];
    a.gam = h->pp.gam[0];
    a.gam_1 = h->pp.gam_1[0];
    a.cfl_glm = h->cfg.cfl_glm;
    a.ib = h->ib;
    for (int d = 0; d < 3; ++d) {
        a.has_dir[d] = 0;
        for (const auto& b : h->blocks) a.has_dir[d] |= b.n[d] > 1;
    }
    const int nb = (int)h->blocks.size();
    long long most = 1;
    for (auto& b : h->blocks) most = std::max(most, ((long long)b.n[0] * b.n[1] * b.n[2] + 1023) / 1024);
    PK_CUDA(h, cudaMemsetAsync(h->d_ch, 0, sizeof(unsigned long long), h->stream));
    k_chspeed_blocks<<<dim3((unsigned)std::min<long long>(most, 1024), nb), 256, 0, h->stream>>>(h->d_desc[h->cur], a,
                                                                                              h->d_ch);
    PK_CUDA(h, cudaGetLastError());
    h->launches += 1;
    unsigned long long bits = 0;
    PK_CUDA(h, cudaMemcpyAsync(&bits, h->d_ch, sizeof bits, cudaMemcpyDeviceToHost, h->stream));
    PK_CUDA(h, cudaStreamSynchronize(h->stream));
    double c = 1.1754943508222875e-38;                // chspeed = small (:112), then max over the cells
    double x;
    std::memcpy(&x, &bits, sizeof x);
    if (bits) c = (x > c) ? x : c;
    if (h->reduce_cb) c = h->reduce_cb(h->comm_ctx, c, 1);   // piernik_MPI_Allreduce(chspeed, pMAX)
    *ch = c;
    return PK_OK;
}

int glm_scalars_for(pk_ctx* h, double dt, double ch_now, double* ch, double* fac)
{
    int eff;
    const double mdl = min_dl(h, &eff);
    *ch = ch_now;
    *fac = 1.0;
    if (!h->cfg.magnetic) return PK_OK;
    double c = DBL_MAX;
    if (!h->cfg.ch_grid) {
        if (int rc = gas_chspeed(h, &c)) return rc;
    } else {
        if (eff) {
            const double x = (h->cfg.cfl_glm * mdl) / dt;
            c = (x < c) ? x : c;
        }
        if (h->reduce_cb) c = h->reduce_cb(h->comm_ctx, c, 0);   // piernik_MPI_Allreduce(chspeed, pMIN) (hdc.F90:138)
    }
    double f = 0.0;
    if (eff) {
        const double x = (h->cfg.glm_alpha * c) / (mdl / dt);
        f = (x > f) ? x : f;
    }
    *ch = c;
    *fac = std::exp(-f);
    if (h->reduce_cb) *fac = h->reduce_cb(h->comm_ctx, *fac, 0);   // piernik_MPI_Allreduce(fac, pMIN) (:333)
    return PK_OK;
}

int glm_scalars(pk_ctx* h, double dt, double* ch, double* fac) { return glm_scalars_for(h, dt, h->ts.chspeed, ch, fac); }

// the glmdamping factor for chspeed ch over dt_eff (hdc.F90:310-332)
double glm_fac_for(pk_ctx* h, double dt_eff, double ch)
{
    int eff;
    const double mdl = min_dl(h, &eff);
    double f = 0.0;
    if (eff) {
        const double x = (h->cfg.glm_alpha * ch) / (mdl / dt_eff);
        f = (x > f) ? x : f;
    }
    const double fac = std::exp(-f);
    return h->reduce_cb ? h->reduce_cb(h->comm_ctx, fac, 0) : fac;   // pMIN over ranks (hdc.F90:333)
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------

extern "C" {

int pk_abi_version(void) { return PK_ABI_VERSION; }

void pk_config_default(pk_config* c)
{
    std::memset(c, 0, sizeof(*c));
    c->nfluids = 1;
    c->fluid_kind[0] = PK_FLUID_ION;
    c->gamma[0] = c->gamma[1] = c->gamma[2] = 5.0 / 3.0;
    c->magnetic = 1;
    c->limiter = PK_LIM_VANLEER;       // global.F90:209
    c->limiter_b = PK_LIM_VANLEER;     // limiter_b = limiter
    c->use_smalld = 1;
    c->use_smallei = 1;
    c->disallow_negatives = 1;
    c->smalld = 1.0e-3;                // the reference auto-sets it from the minimum density when left unset
    c->smallei = 1.0e-10;
    c->cfl = 0.7;
    c->cfl_glm = 0.7;
    c->glm_alpha = 0.1;
    c->integration_order = 2;
    c->nb = 4;
    c->dt_initial = -1.0;
    c->dt_max_grow = 2.0;
    c->dt_min = DBL_MIN;
    c->dt_max = DBL_MAX;
    c->tend = DBL_MAX;
    c->cflcontrol = PK_CFL_REDO;       // global.F90:218
    c->cfl_max = 0.9;                  // :233
    c->dt_shrink = 0.5;                // :245
    c->max_redostep_attempts = 10;     // :258
    c->interpolation = PK_INTERP_LINEAR;   // :220
    c->solver = PK_SOLVER_SPLIT;          // :423-437
    c->ord_fluid_prolong = 0;             // O_INJ (:260)
    c->ord_mag_prolong = 2;               // O_I2 (:259)
    c->w_epsilon = 1.0e-10;            // :255
    c->ch_grid = 1;                    // :254
    c->use_eglm = 0;                   // :252
}

int pk_create(const pk_config* cfg, pk_handle* out)
{
    if (cfg && (cfg->cflcontrol < PK_CFL_NONE || cfg->cflcontrol > PK_CFL_AUTO || cfg->max_redostep_attempts < 0 ||
                cfg->ch_grid < 0 || cfg->ch_grid > 1 || cfg->use_eglm < 0 || cfg->use_eglm > 1 ||
                cfg->interpolation < PK_INTERP_LINEAR || cfg->interpolation > PK_INTERP_WENO3 ||
                cfg->solver < PK_SOLVER_SPLIT || cfg->solver > PK_SOLVER_UNSPLIT ||
                (cfg->use_eglm && cfg->solver != PK_SOLVER_SPLIT)))   // hdc.F90:388: eglm needs RIEMANN_SPLIT
        return PK_E_ARG;
    if (!cfg || !out) return PK_E_ARG;
    *out = nullptr;
    const pk_config& c = *cfg;
    bool ok = c.nfluids >= 1 && c.nfluids <= 3 && c.nb >= 2 && c.cfl > 0.0 && c.cfl <= 1.0 &&
              (c.integration_order == 1 || c.integration_order == 2) && c.limiter >= 0 && c.limiter <= 3 &&
              c.limiter_b >= 0 && c.limiter_b <= 3;
    for (int f = 0; ok && f < c.nfluids; ++f)
        if (c.fluid_kind[f] < 0 || c.fluid_kind[f] > 2 || (f > 0 && c.fluid_kind[f] <= c.fluid_kind[f - 1])) ok = false;
    if (!ok) return PK_E_ARG;
    // structure of the fluid set: energy fluids then dust; the ionized fluid carries B
    const int ndst = (c.fluid_kind[c.nfluids - 1] == PK_FLUID_DST) ? 1 : 0;
    const int nen = c.nfluids - ndst;
    int phys;
    if (!c.magnetic && nen == 1 && ndst == 0) phys = 0;
    else if (!c.magnetic && nen == 1 && ndst == 1) phys = 1;
    else if (c.magnetic && c.fluid_kind[0] == PK_FLUID_ION && nen == 1 && ndst == 0) phys = 2;
    else if (c.magnetic && c.fluid_kind[0] == PK_FLUID_ION && nen == 2 && ndst == 0) phys = 3;
    else if (c.magnetic && c.fluid_kind[0] == PK_FLUID_ION && nen == 2 && ndst == 1) phys = 4;
    else return PK_E_UNSUPPORTED;
    // prolongation orders of refined domains (cg_list_global.F90:195-207,
    // global.F90:561-566: fluids other than injection / linear degrade to injection)
    ProlongCoef pro_u, pro_b;
    const int ofl = (c.ord_fluid_prolong == 0 || c.ord_fluid_prolong == 1) ? c.ord_fluid_prolong : 0;
    if (!prolong_coef(ofl, &pro_u) || !prolong_coef(c.ord_mag_prolong, &pro_b)) return PK_E_ARG;
    if (2 * pro_u.r > c.nb || (c.magnetic && 2 * pro_b.r > c.nb)) return PK_E_ARG;

    pk_ctx* h = new pk_ctx();
    h->cfg = c;
    h->cfg.ord_fluid_prolong = ofl;
    h->pro_u = pro_u;
    h->pro_b = pro_b;
    h->phys = phys;
    int nvf = 0;
    for (int f = 0; f < c.nfluids; ++f) {
        nvf += (c.fluid_kind[f] == PK_FLUID_DST) ? 4 : 5;
        h->pp.gam[f] = (c.fluid_kind[f] == PK_FLUID_DST) ? -1.0 : c.gamma[f];
        h->pp.gam_1[f] = h->pp.gam[f] - 1.0;
        h->pp.rgam_1[f] = 1.0 / h->pp.gam_1[f];
        h->pp.rgam[f] = 1.0 / h->pp.gam[f];
    }
    h->nvf = nvf;
    h->ib = nvf;
    h->nplanes = nvf + (c.magnetic ? 4 : 0);
    h->pp.smalld = c.smalld;
    h->pp.smallei = c.smallei;
    h->pp.use_smalld = c.use_smalld;
    h->pp.use_smallei = c.use_smallei;
    h->pp.disallow_negatives = c.disallow_negatives;
    h->pp.lim = c.limiter;
    h->pp.limb = c.limiter_b;
    h->pp.weno3 = c.interpolation == PK_INTERP_WENO3;
    h->pp.w_epsilon = c.w_epsilon;
    std::memset(&h->ts, 0, sizeof(h->ts));
    h->ts.dt_old = -1.0;
    h->ts.dt_cur_shrink = 1.0;                        // global.F90:571
    h->ts.cfl_c = 1.0;                                // timestep_pub.F90:42
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc(&h->d_status, sizeof(unsigned)) != cudaSuccess ||
        cudaMemset(h->d_status, 0, sizeof(unsigned)) != cudaSuccess ||
        cudaMalloc(&h->d_counter, 8 * sizeof(unsigned)) != cudaSuccess ||
        cudaMalloc(&h->d_step, sizeof(StepParams)) != cudaSuccess ||
        cudaMallocHost(&h->h_step, sizeof(StepParams)) != cudaSuccess || ops_of(h)->prepare(h) != PK_OK) {
        delete h;
        return PK_E_CUDA;
    }
    *out = h;
    return PK_OK;
}

int pk_destroy(pk_handle h)
{
    if (!h) return PK_E_ARG;
    cudaStreamSynchronize(h->stream);
    invalidate_graph(h);
    for (auto& b : h->blocks) {
        cudaFree(b.buf[0]);
        cudaFree(b.buf[1]);
        cudaFree(b.uh);
        cudaFree(b.stage);
        for (int d = 0; d < 3; ++d) cudaFree(b.flux[d]);
        cudaFree(b.flag);
    }
    for (auto& p : h->ev_used) { cudaEventDestroy(p.first); cudaEventDestroy(p.second); }
    for (auto& p : h->ev_free) { cudaEventDestroy(p.first); cudaEventDestroy(p.second); }
    for (int d = 0; d < 3; ++d) {
        cudaFree(h->batch[d].dev);
        for (StageList& s : h->sbatch[d]) cudaFree(s.dev);
        cudaFree(h->rdev[d]);
    }
    cudaFree(h->d_rcount);
    cudaFree(h->d_eglm);
    for (double* p : h->grad_ckpt) cudaFree(p);
    for (double* p : h->grad_pool) cudaFree(p);
    for (double* p : h->grad_star) cudaFree(p);
    for (unsigned short* p : h->grad_flags) cudaFree(p);
    cudaFree(h->lam);
    cudaFree(h->lam_tmp);
    cudaFree(h->lam_m1);
    free_segs(h);
    free_levels(h);
    cudaFree(h->d_xptr[0]);
    cudaFree(h->d_xptr[1]);
    for (auto& b : h->blocks) cudaFree(b.retry);
    cudaFree(h->d_inst[0]);
    cudaFree(h->d_inst[1]);
    cudaFree(h->d_desc[0]);
    cudaFree(h->d_desc[1]);
    cudaFree(h->d_status);
    cudaFree(h->d_counter);
    cudaFree(h->d_red);
    cudaFree(h->d_ch);
    cudaFree(h->d_step);
    cudaFreeHost(h->h_red);
    cudaFreeHost(h->h_step);
    cudaStreamDestroy(h->stream);
    delete h;
    return PK_OK;
}

const char* pk_last_error(pk_handle h) { return h ? h->err.c_str() : "null handle"; }

void* pk_stream(pk_handle h) { return h ? (void*)h->stream : nullptr; }

int pk_block_add(pk_handle h, const int32_t n[3], const double dl[3], const int32_t bnd[6], int32_t* id_out)
{
    if (!h || !n || !dl || !bnd) return PK_E_ARG;
    if (h->ninst > 1) return fail(h, PK_E_STATE, "stacked instances live in one block");
    Block b;
    for (int d = 0; d < 3; ++d) {
        if (n[d] < 1 || !(dl[d] > 0.0)) return fail(h, PK_E_ARG, "block extent and cell size must be positive");
        b.n[d] = n[d];
        b.g[d] = n[d] > 1 ? h->cfg.nb : 0;
        b.ext[d] = n[d] + 2 * b.g[d];
        b.dl[d] = dl[d];
        for (int s = 0; s < 2; ++s) {
            b.bnd[d][s] = bnd[2 * d + s];
            if (b.bnd[d][s] < 0 || b.bnd[d][s] > 2) return fail(h, PK_E_ARG, "unknown boundary type");
        }
        if (n[d] > 1 && n[d] < h->cfg.nb && b.bnd[d][0] == PK_BND_PER)
            return fail(h, PK_E_ARG, "periodic direction shorter than the guard width");
        if (!h->blocks.empty() && ((h->blocks[0].n[d] > 1) != (n[d] > 1)))
            return fail(h, PK_E_ARG, "all blocks must have the same directions (dom%has_dir)");
    }
    if (h->cfg.magnetic)
        for (int d = 0; d < 3; ++d)
            if (b.n[d] > 1 && (b.bnd[d][0] != PK_BND_PER || b.bnd[d][1] != PK_BND_PER))
                return fail(h, PK_E_UNSUPPORTED, "magnetised blocks support periodic boundaries only");
    b.plane = (long long)b.ext[0] * b.ext[1] * b.ext[2];
    double* p = nullptr;
    if (cudaMalloc(&p, sizeof(double) * h->nplanes * b.plane) != cudaSuccess)
        return fail(h, PK_E_NOMEM, "cudaMalloc of the block state failed");
    PK_CUDA(h, cudaMemsetAsync(p, 0, sizeof(double) * h->nplanes * b.plane, h->stream));
    b.buf[h->cur] = p;                      // the state lives in the current parity's buffer
    h->blocks.push_back(b);
    h->batch_dirty = true;
    h->x_dirty = true;
    h->x_ptrs_dirty = true;
    invalidate_graph(h);
    if (id_out) *id_out = (int32_t)h->blocks.size() - 1;
    const int need = (int)h->blocks.size() * 12;
    if (need > h->red_cap) {
        PK_CUDA(h, cudaStreamSynchronize(h->stream));
        cudaFree(h->d_red);
        cudaFreeHost(h->h_red);
        h->red_cap = need + 1200;
        PK_CUDA(h, cudaMalloc(&h->d_red, sizeof(unsigned long long) * h->red_cap));
        PK_CUDA(h, cudaMallocHost(&h->h_red, sizeof(unsigned long long) * h->red_cap));
    }
    return PK_OK;
}

int pk_block_remove(pk_handle h, int32_t id)
{
    if (!h) return PK_E_ARG;
    if (id < 0 || id >= (int)h->blocks.size()) return fail(h, PK_E_ARG, "unknown block id");
    if (h->ninst > 1) return fail(h, PK_E_STATE, "stacked instances live in one block");
    if (!h->grad_ckpt.empty() || h->lam) return fail(h, PK_E_STATE, "release the differentiable path first (pk_grad_release)");
    PK_CUDA(h, cudaStreamSynchronize(h->stream));
    invalidate_graph(h);
    Block& b = h->blocks[id];
    cudaFree(b.buf[0]);
    cudaFree(b.buf[1]);
    cudaFree(b.uh);
    cudaFree(b.stage);
    cudaFree(b.retry);
    cudaFree(b.leaf);
    cudaFree(b.flag);
    for (int d = 0; d < 3; ++d) cudaFree(b.flux[d]);
    h->blocks.erase(h->blocks.begin() + id);
    h->batch_dirty = true;
    h->x_dirty = true;
    h->x_ptrs_dirty = true;
    return PK_OK;
}

static int get_block(pk_ctx* h, int id, Block** b)
{
    if (!h) return PK_E_ARG;
    if (id < 0 || id >= (int)h->blocks.size()) return fail(h, PK_E_ARG, "unknown block id");
    *b = &h->blocks[id];
    return PK_OK;
}

int pk_upload(pk_handle h, int32_t id, const double* u, const double* bf, const double* psi, int32_t layout)
{
    Block* b;
    if (int rc = get_block(h, id, &b)) return rc;
    if (!u || (h->cfg.magnetic && (!bf || !psi))) return fail(h, PK_E_ARG, "null array");
    const long long nc = b->plane;
    double* s = state(h, *b);
    if (layout == PK_LAYOUT_SOA) {
        PK_CUDA(h, cudaMemcpyAsync(s, u, sizeof(double) * h->nvf * nc, cudaMemcpyHostToDevice, h->stream));
        if (h->cfg.magnetic) {
            PK_CUDA(h, cudaMemcpyAsync(s + (long long)h->ib * nc, bf, sizeof(double) * 3 * nc, cudaMemcpyHostToDevice, h->stream));
            PK_CUDA(h, cudaMemcpyAsync(s + (long long)(h->ib + 3) * nc, psi, sizeof(double) * nc, cudaMemcpyHostToDevice, h->stream));
        }
    } else if (layout == PK_LAYOUT_FORTRAN) {
        if (!b->stage) PK_CUDA(h, cudaMalloc(&b->stage, sizeof(double) * h->nvf * nc));
        PK_CUDA(h, cudaMemcpyAsync(b->stage, u, sizeof(double) * h->nvf * nc, cudaMemcpyHostToDevice, h->stream));
        k_aos_to_soa<<<grid1d(nc, 256), 256, 0, h->stream>>>(b->stage, s, nc, h->nvf, 0, nc);
        PK_CUDA(h, cudaGetLastError());
        h->launches += 1;
        if (h->cfg.magnetic) {
            // the staging buffer is reused once the first conversion has run (same stream)
            PK_CUDA(h, cudaMemcpyAsync(b->stage, bf, sizeof(double) * 3 * nc, cudaMemcpyHostToDevice, h->stream));
            k_aos_to_soa<<<grid1d(nc, 256), 256, 0, h->stream>>>(b->stage, s, nc, 3, h->ib, nc);
            PK_CUDA(h, cudaGetLastError());
            h->launches += 1;
            PK_CUDA(h, cudaMemcpyAsync(s + (long long)(h->ib + 3) * nc, psi, sizeof(double) * nc, cudaMemcpyHostToDevice, h->stream));
        }
    } else {
        return fail(h, PK_E_ARG, "unknown layout");
    }
    b->guards_stale = false;
    return PK_OK;
}

int pk_download(pk_handle h, int32_t id, double* u, double* bf, double* psi, int32_t layout)
{
    Block* b;
    if (int rc = get_block(h, id, &b)) return rc;
    if (!u || (h->cfg.magnetic && (!bf || !psi))) return fail(h, PK_E_ARG, "null array");
    if (b->guards_stale)
        if (int rc = refresh_guards(h, *b)) return rc;
    const long long nc = b->plane;
    double* s = state(h, *b);
    if (layout == PK_LAYOUT_SOA) {
        PK_CUDA(h, cudaMemcpyAsync(u, s, sizeof(double) * h->nvf * nc, cudaMemcpyDeviceToHost, h->stream));
        if (h->cfg.magnetic) {
            PK_CUDA(h, cudaMemcpyAsync(bf, s + (long long)h->ib * nc, sizeof(double) * 3 * nc, cudaMemcpyDeviceToHost, h->stream));
            PK_CUDA(h, cudaMemcpyAsync(psi, s + (long long)(h->ib + 3) * nc, sizeof(double) * nc, cudaMemcpyDeviceToHost, h->stream));
        }
    } else if (layout == PK_LAYOUT_FORTRAN) {
        if (!b->stage) PK_CUDA(h, cudaMalloc(&b->stage, sizeof(double) * h->nvf * nc));
        k_soa_to_aos<<<grid1d(nc, 256), 256, 0, h->stream>>>(s, b->stage, nc, h->nvf, 0, nc);
        PK_CUDA(h, cudaGetLastError());
        h->launches += 1;
        PK_CUDA(h, cudaMemcpyAsync(u, b->stage, sizeof(double) * h->nvf * nc, cudaMemcpyDeviceToHost, h->stream));
        if (h->cfg.magnetic) {
            PK_CUDA(h, cudaStreamSynchronize(h->stream));   // the staging buffer is reused for b
            k_soa_to_aos<<<grid1d(nc, 256), 256, 0, h->stream>>>(s, b->stage, nc, 3, h->ib, nc);
            PK_CUDA(h, cudaGetLastError());
            h->launches += 1;
            PK_CUDA(h, cudaMemcpyAsync(bf, b->stage, sizeof(double) * 3 * nc, cudaMemcpyDeviceToHost, h->stream));
            PK_CUDA(h, cudaMemcpyAsync(psi, s + (long long)(h->ib + 3) * nc, sizeof(double) * nc, cudaMemcpyDeviceToHost, h->stream));
        }
    } else {
        return fail(h, PK_E_ARG, "unknown layout");
    }
    PK_CUDA(h, cudaStreamSynchronize(h->stream));
    return PK_OK;
}

int pk_solve_cg(pk_handle h, int32_t id, int32_t ddim, int32_t istep, double dt, double chspeed)
{
    Block* b;
    if (int rc = get_block(h, id, &b)) return rc;
    if (ddim < 1 || ddim > 3) return fail(h, PK_E_ARG, "ddim must be 1..3");
    const int dir = ddim - 1;
    double rk;
    int first;
    if (istep == PK_EULER) { rk = 1.0; first = 1; }
    else if (istep == PK_RK2_1) { rk = 0.5; first = 1; }
    else if (istep == PK_RK2_2) { rk = 1.0; first = 0; }
    else return fail(h, PK_E_ARG, "istep must be PK_EULER, PK_RK2_1 or PK_RK2_2");
    if (b->n[dir] <= 1) return PK_OK;
    if (b->guards_stale)
        if (int rc = fill_guards_block(h, *b)) return rc;
    if (!b->uh) PK_CUDA(h, cudaMalloc(&b->uh, sizeof(double) * h->nplanes * b->plane));
    if (stage_chunked(*b, dir))
        if (int rc = ensure_pingpong(h)) return rc;
    if (int rc = put_step_params(h, dt, chspeed, 1.0)) return rc;   // rk_coef(istep) * dt / cg%dl(ddim) on the device
    return ops_of(h)->stage(h, *b, dir, first, rk);
}

int pk_fill_guards(pk_handle h)
{
    if (!h) return PK_E_ARG;
    for (auto& b : h->blocks)
        if (int rc = fill_guards_block(h, b)) return rc;
    return exchange_guards(h);
}

int pk_set_instances(pk_handle h, int32_t count)
{
    if (!h || count < 1) return PK_E_ARG;
    if (h->blocks.size() != 1) return fail(h, PK_E_UNSUPPORTED, "instances are stacked in one block");
    Block& b = h->blocks[0];
    if (count > 1) {
        if (b.n[2] % count) return fail(h, PK_E_ARG, "the z extent must be a multiple of the instance count");
        const int seg = b.n[2] / count;
        if (seg < h->cfg.nb || seg > 256) return fail(h, PK_E_ARG, "instances need nb..256 cells along z");
        for (int d = 0; d < 3; ++d)
            if (b.n[d] > 1 && (b.bnd[d][0] != PK_BND_PER || b.bnd[d][1] != PK_BND_PER))
                return fail(h, PK_E_UNSUPPORTED, "stacked instances are periodic in every direction");
        if (h->cfg.integration_order != 2 || h->connected || h->cfg.cflcontrol == PK_CFL_REDO ||
            h->cfg.cflcontrol == PK_CFL_FLEX || !h->cfg.ch_grid)
            return fail(h, PK_E_UNSUPPORTED,
                        "stacked instances need RK2, one unconnected block, no step retry and ch_grid = 1");
        b.seg_len = seg;
    } else {
        b.seg_len = 0;
    }
    PK_CUDA(h, cudaStreamSynchronize(h->stream));
    cudaFree(h->d_step);
    cudaFreeHost(h->h_step);
    h->d_step = nullptr;
    h->h_step = nullptr;
    PK_CUDA(h, cudaMalloc(&h->d_step, sizeof(StepParams) * count));
    PK_CUDA(h, cudaMallocHost(&h->h_step, sizeof(StepParams) * count));
    h->ninst = count;
    h->its.assign(count, h->ts);
    if (count * 12 > h->red_cap) {
        cudaFree(h->d_red);
        cudaFreeHost(h->h_red);
        h->red_cap = count * 12 + 1200;
        PK_CUDA(h, cudaMalloc(&h->d_red, sizeof(unsigned long long) * h->red_cap));
        PK_CUDA(h, cudaMallocHost(&h->h_red, sizeof(unsigned long long) * h->red_cap));
    }
    // the instances as blocks for the CFL reduction, one table per parity
    if (int rc = ensure_pingpong(h)) return rc;
    for (int p = 0; p < 2; ++p) {
        cudaFree(h->d_inst[p]);
        h->d_inst[p] = nullptr;
        if (count < 2) continue;
        std::vector<BlockDesc> t(count);
        for (int i = 0; i < count; ++i) {
            BlockDesc& d = t[i];
            d.in = b.buf[p] + (long long)i * b.seg_len * b.ext[0] * b.ext[1];
            d.out = nullptr;
            d.plane = b.plane;
            for (int k = 0; k < 3; ++k) {
                d.ext[k] = b.ext[k];
                d.g[k] = b.g[k];
                d.n[k] = b.n[k];
                d.dl[k] = b.dl[k];
            }
            d.n[2] = b.seg_len;
            d.wrap = 1;
        }
        PK_CUDA(h, cudaMalloc(&h->d_inst[p], sizeof(BlockDesc) * count));
        PK_CUDA(h, cudaMemcpy(h->d_inst[p], t.data(), sizeof(BlockDesc) * count, cudaMemcpyHostToDevice));
    }
    invalidate_graph(h);
    return PK_OK;
}

int pk_get_instance_state(pk_handle h, int32_t i, pk_time_state* st)
{
    if (!h || !st || i < 0 || i >= h->ninst) return PK_E_ARG;
    *st = h->ninst > 1 ? h->its[i] : h->ts;
    return PK_OK;
}

int pk_set_instance_state(pk_handle h, int32_t i, const pk_time_state* st)
{
    if (!h || !st || i < 0 || i >= h->ninst) return PK_E_ARG;
    if (h->ninst > 1) h->its[i] = *st;
    if (i == 0) h->ts = *st;
    return PK_OK;
}

int pk_set_domain(pk_handle h, const int64_t ncells[3], const int32_t periodic[3])
{
    if (!h || !ncells || !periodic) return PK_E_ARG;
    for (int d = 0; d < 3; ++d)
        if (ncells[d] < 1) return fail(h, PK_E_ARG, "domain extents must be positive");
    for (int d = 0; d < 3; ++d) {
        h->dom[d] = ncells[d];
        h->dom_periodic[d] = periodic[d] ? 1 : 0;
    }
    h->connected = true;
    h->x_dirty = true;
    h->batch_dirty = true;
    invalidate_graph(h);
    return PK_OK;
}

int pk_block_remote(pk_handle h, int32_t owner, const int32_t n[3], const int64_t off[3])
{
    if (!h || !n || !off) return PK_E_ARG;
    if (owner < 0) return fail(h, PK_E_ARG, "owner rank must be >= 0");
    RemoteBlock r;
    r.owner = owner;
    for (int d = 0; d < 3; ++d) {
        if (n[d] < 1) return fail(h, PK_E_ARG, "block extent must be positive");
        if (!h->blocks.empty() && ((h->blocks[0].n[d] > 1) != (n[d] > 1)))
            return fail(h, PK_E_ARG, "all blocks must have the same directions (dom%has_dir)");
        r.n[d] = n[d];
        r.off[d] = off[d];
    }
    h->remote.push_back(r);
    h->x_dirty = true;
    return PK_OK;
}

int pk_halo_peers(pk_handle h, int32_t* peers, int32_t max_peers, int32_t* count)
{
    if (!h || !count) return PK_E_ARG;
    if (int rc = exchange_prepare(h)) return rc;
    *count = (int32_t)h->xpeers.size();
    for (int i = 0; i < (int)h->xpeers.size() && i < max_peers; ++i)
        if (peers) peers[i] = h->xpeers[i].rank;
    return PK_OK;
}

static XPeerDev* find_peer(pk_ctx* h, int peer)
{
    for (auto& p : h->xpeers)
        if (p.rank == peer) return &p;
    return nullptr;
}

// the segment lists of one peer for the exchange before a sweep along dir (-1: every guard cell)
static int peer_lists(pk_ctx* h, int peer, int dir, const XSegList** send, const XSegList** recv)
{
    if (dir < -1 || dir > 2) return fail(h, PK_E_ARG, "dir must be -1..2");
    if (int rc = exchange_prepare(h)) return rc;
    XPeerDev* p = find_peer(h, peer);
    if (!p) return fail(h, PK_E_ARG, "no halo traffic with that rank");
    if (dir >= 0 && !h->x_dir) return fail(h, PK_E_UNSUPPORTED, "per-direction halos need a single-level domain");
    *send = dir < 0 ? &p->send : &p->send_dir[dir];
    *recv = dir < 0 ? &p->recv : &p->recv_dir[dir];
    return PK_OK;
}

int pk_halo_sizes_dir(pk_handle h, int32_t peer, int32_t dir, int64_t* send_doubles, int64_t* recv_doubles)
{
    if (!h) return PK_E_ARG;
    const XSegList *s, *r;
    if (int rc = peer_lists(h, peer, dir, &s, &r)) return rc;
    if (send_doubles) *send_doubles = s->total * h->nplanes;
    if (recv_doubles) *recv_doubles = r->total * h->nplanes;
    return PK_OK;
}

int pk_halo_sizes(pk_handle h, int32_t peer, int64_t* send_doubles, int64_t* recv_doubles)
{
    return pk_halo_sizes_dir(h, peer, -1, send_doubles, recv_doubles);
}

// sync: wait for the copy (the whole-halo calls); the per-direction calls
// stay in the handle's stream order for a transport that follows it
static int halo_copy(pk_ctx* h, int peer, int dir, double* buf, int to_buf, bool sync)
{
    const XSegList *s, *r;
    if (int rc = peer_lists(h, peer, dir, &s, &r)) return rc;
    if (!buf && (to_buf ? s : r)->total > 0) return fail(h, PK_E_ARG, "null buffer");
    const XSegList& l = to_buf ? *s : *r;
    if (l.total > 0) {
        k_halo_copy<<<grid1d(l.total, 256), 256, 0, h->stream>>>(l.dev, l.n, l.total, h->d_xptr[h->cur], h->nplanes, buf,
                                                                to_buf);
        PK_CUDA(h, cudaGetLastError());
        h->launches += 1;
    }
    if (sync) PK_CUDA(h, cudaStreamSynchronize(h->stream));
    return PK_OK;
}

int pk_halo_pack(pk_handle h, int32_t peer, double* sendbuf_dev)
{
    if (!h) return PK_E_ARG;
    return halo_copy(h, peer, -1, sendbuf_dev, 1, true);
}

int pk_halo_unpack(pk_handle h, int32_t peer, const double* recvbuf_dev)
{
    if (!h) return PK_E_ARG;
    return halo_copy(h, peer, -1, const_cast<double*>(recvbuf_dev), 0, true);
}

int pk_halo_pack_dir(pk_handle h, int32_t peer, int32_t dir, double* sendbuf_dev)
{
    if (!h) return PK_E_ARG;
    return halo_copy(h, peer, dir, sendbuf_dev, 1, false);
}

int pk_halo_unpack_dir(pk_handle h, int32_t peer, int32_t dir, const double* recvbuf_dev)
{
    if (!h) return PK_E_ARG;
    return halo_copy(h, peer, dir, const_cast<double*>(recvbuf_dev), 0, false);
}

int pk_set_comm(pk_handle h, pk_halo_fn halo, pk_reduce_fn reduce, void* ctx)
{
    if (!h) return PK_E_ARG;
    h->halo_cb = halo;
    h->reduce_cb = reduce;
    h->comm_ctx = ctx;
    invalidate_graph(h);
    return PK_OK;
}

int pk_block_place(pk_handle h, int32_t id, const int64_t off[3])
{
    return pk_block_place_level(h, id, 0, off);
}

int pk_block_place_level(pk_handle h, int32_t id, int32_t level, const int64_t off[3])
{
    Block* b;
    if (int rc = get_block(h, id, &b)) return rc;
    if (!off) return fail(h, PK_E_ARG, "null offset");
    if (level < 0 || level > 8) return fail(h, PK_E_ARG, "level must lie in 0..8");
    if (level > 0 && h->ninst > 1) return fail(h, PK_E_STATE, "stacked instances are not refined");
    for (int d = 0; d < 3; ++d) b->off[d] = off[d];
    b->level = level;
    b->placed = true;
    h->x_dirty = true;
    h->batch_dirty = true;
    invalidate_graph(h);
    return PK_OK;
}

int pk_sweep(pk_handle h, int32_t cdim, double dt, double chspeed)
{
    if (!h) return PK_E_ARG;
    if (cdim < 1 || cdim > 3) return fail(h, PK_E_ARG, "cdim must be 1..3");
    if (int rc = put_step_params(h, dt, chspeed, 1.0)) return rc;
    return sweep_impl(h, cdim - 1, dt, chspeed, 0, 1.0);
}

int pk_glm_damp(pk_handle h, double fac)
{
    if (!h) return PK_E_ARG;
    if (!h->cfg.magnetic) return PK_OK;
    return glm_scale(h, fac);
}

int pk_timestep_raw(pk_handle h, double* dt_out, double* c_all_out)
{
    if (!h) return PK_E_ARG;
    if (h->blocks.empty()) return fail(h, PK_E_STATE, "no block registered");
    if (int rc = exchange_prepare(h)) return rc;       // a refined domain's leaf masks
    const int nb = (int)h->blocks.size();
    PK_CUDA(h, cudaMemsetAsync(h->d_red, 0, sizeof(unsigned long long) * 12 * nb, h->stream));
    CflArgs a;
    a.nfl = h->cfg.nfluids;
    int beg = 0;
    for (int f = 0; f < 3; ++f) {
        a.fl[f].kind = f < a.nfl ? h->cfg.fluid_kind[f] : K_NONE;
        a.fl[f].beg = beg;
        a.fl[f].gam = h->pp.gam[f];
        a.fl[f].gam_1 = h->pp.gam_1[f];
        if (f < a.nfl) beg += (h->cfg.fluid_kind[f] == PK_FLUID_DST) ? 4 : 5;
    }
    a.magnetic = h->cfg.magnetic;
    a.ib = h->ib;
    if (nb > 1) {
        if (int rc = build_batch(h)) return rc;
        long long most = 1;                               // about four cells per thread in the largest block
        for (auto& b : h->blocks) most = std::max(most, ((long long)b.n[0] * b.n[1] * b.n[2] + 1023) / 1024);
        dim3 grid((unsigned)std::min<long long>(most, 1024), nb);
        k_cfl_blocks<<<grid, 256, 0, h->stream>>>(h->d_desc[h->cur], a, h->d_red);
        PK_CUDA(h, cudaGetLastError());
        h->launches += 1;
    } else {
        Block& b = h->blocks[0];
        const long long ncell = (long long)b.n[0] * b.n[1] * b.n[2];
        k_cfl<<<grid1d(ncell, 256), 256, 0, h->stream>>>(box_of(b), state(h, b), a, h->d_red);
        PK_CUDA(h, cudaGetLastError());
        h->launches += 1;
    }
    PK_CUDA(h, cudaMemcpyAsync(h->h_red, h->d_red, sizeof(unsigned long long) * 12 * nb, cudaMemcpyDeviceToHost, h->stream));
    PK_CUDA(h, cudaStreamSynchronize(h->stream));
    double dt = DBL_MAX, c_all = 0.0;                  // timestep.F90:161-162
    for (int i = 0; i < nb; ++i) {
        const Block& b = h->blocks[i];
        if (b.leaf_cells == 0) continue;               // wholly covered by finer blocks
        for (int f = 0; f < h->cfg.nfluids; ++f) {
            double cm[4];
            for (int d = 0; d < 4; ++d) {
                unsigned long long bits = h->h_red[12 * i + 4 * f + d];
                std::memcpy(&cm[d], &bits, sizeof(double));
            }
            double dtp[3];
            for (int d = 0; d < 3; ++d) dtp[d] = (b.n[d] > 1 && cm[d] > 0.0) ? b.dl[d] / cm[d] : DBL_MAX;
            double m = dtp[0];
            m = (dtp[1] < m) ? dtp[1] : m;
            m = (dtp[2] < m) ? dtp[2] : m;
            const double dtf = h->cfg.cfl * m;         // :493
            dt = (dtf < dt) ? dtf : dt;
            c_all = (cm[3] > c_all) ? cm[3] : c_all;
        }
    }
    if (dt_out) *dt_out = dt;
    if (c_all_out) *c_all_out = c_all;
    return PK_OK;
}

// the sanity factors of time_step (timestep.F90:200-228) on a raw dt for one
// time state; returns PK_E_DTMIN when dt < dt_min
// cfl_auto (timestep.F90:368-405), the cfl_manager of cflcontrol = 'auto' in
// the main time_step call: scales dt by cfl_c, a running factor that follows
// the change of the signal speed c_all and of dt between steps.  (In the
// reference the routine scales the module's dt while time_step holds it as
// its dummy argument; this is the intended effect, dt x cfl_c.)
static void cfl_auto(const pk_config& c, pk_time_state& ts, double& dt, double c_all)
{
    double cfl_c = ts.cfl_c > 0.0 ? ts.cfl_c : 1.0;   // an unset state reads as the initial one
    double stepcfl_old = ts.stepcfl;
    double stepcfl = c.cfl;
    if (ts.c_all_old > 0.0) stepcfl = (c_all / ts.c_all_old) * c.cfl;
    else stepcfl_old = c.cfl;
    if (stepcfl > 0.0 && ts.dt_old > 0.0) {
        double r = ((stepcfl_old / stepcfl) * dt) / ts.dt_old;
        r = (r < 1.0) ? r : 1.0;                       // min(one, ...)
        const double x = 0.5 * (cfl_c + r);
        cfl_c = (x < 1.0) ? x : 1.0;
        dt = dt * cfl_c;
    } else {
        cfl_c = 1.0;
    }
    ts.stepcfl = stepcfl;
    ts.cfl_c = cfl_c;
}

static int clamp_dt(const pk_config& c, pk_time_state& ts, double dt, double c_all)
{
    if (ts.nstep < 1) {                               // :200-208
        if (c.dt_initial > 0.0) dt = (c.dt_initial < dt) ? c.dt_initial : dt;
        else if (c.dt_initial < 0.0) {
            const double x = -c.dt_initial * dt;
            dt = (x < dt) ? x : dt;
        }
    } else if (ts.dt_old > 0.0) {
        const double x = ts.dt_old * c.dt_max_grow;
        dt = (x < dt) ? x : dt;
    }
    if (c.cflcontrol == PK_CFL_AUTO) cfl_auto(c, ts, dt, c_all);   // cfl_manager of the main call (:210)
    ts.c_all = c_all;
    if (dt < c.dt_min) {                              // :213-219
        ts.dt = dt;
        return PK_E_DTMIN;
    }
    const double rem = c.tend - ts.t;                 // :221-225
    const double cap = c.solver == PK_SOLVER_UNSPLIT ? rem + ((2.0 * DBL_EPSILON) * rem)
                                                     : (0.5 * rem) + ((2.0 * DBL_EPSILON) * rem);
    dt = (c.dt_max < dt) ? c.dt_max : dt;
    dt = (cap < dt) ? cap : dt;
    ts.dt = dt;
    return PK_OK;
}

// the sweeps of one step, the step scalars already in d_step: replayed from a
// CUDA graph captured once (use_graph) or launched one by one
static int run_step_sweeps(pk_ctx* h, double dt, double ch, double fac)
{
    if (h->use_graph && !h->profiling && !h->halo_cb) {
        if (int rc = exchange_prepare(h)) return rc;
        if (h->blocks.size() > 1)
            if (int rc = build_batch(h)) return rc;   // tables are built outside the capture
        if (int rc = ensure_pingpong(h)) return rc;
        for (auto& b : h->blocks)
            if (!b.uh && !fused_ok(h)) PK_CUDA(h, cudaMalloc(&b.uh, sizeof(double) * h->nplanes * b.plane));
        if (int rc = eglm_alloc(h)) return rc;
        if (!h->graph_exec) {
            // capture the sweeps of one step once; the step scalars are read from d_step
            const int cur0 = h->cur;
            const long long l0 = h->launches;
            PK_CUDA(h, cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
            const int rc = step_sweeps(h, dt, ch, fac);
            h->graph_kernels = h->launches - l0;
            h->launches = l0;                 // counted when the graph is launched
            cudaGraph_t g = nullptr;
            const cudaError_t e = cudaStreamEndCapture(h->stream, &g);
            h->cur = cur0;   // 2 x (number of directions) sweeps: the parity is back where it was
            if (rc) {
                if (g) cudaGraphDestroy(g);
                return rc;
            }
            if (e != cudaSuccess) return fail(h, PK_E_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
            h->graph = g;
            PK_CUDA(h, cudaGraphInstantiate(&h->graph_exec, g, 0));
        }
        PK_CUDA(h, cudaGraphLaunch(h->graph_exec, h->stream));
        h->launches += h->graph_kernels;
        if (fused_ok(h))
            for (auto& b : h->blocks) b.guards_stale = true;
        return PK_OK;
    }
    return step_sweeps(h, dt, ch, fac);
}

// unsplit_sweep (unsplit_sweeps.F90:104-189) of every block: per stage the
// face fluxes of all directions from the stage's input (u, or uh at RK2_2),
// their application to T (uh = u + ... at RK2_1, u itself otherwise) with
// sources and floors, then the boundary update of T.  dt and chspeed come
// from d_step.
static int unsplit_sweep(pk_ctx* h)
{
    const PhysOps* ops = ops_of(h);
    const int order = h->cfg.integration_order, nst = order == 1 ? 1 : 2;
    if (h->connected) {
        // blocks on this device: the stage array uh lives in the other
        // parity's buffer so that the exchange and prolongation tables serve it
        if (!h->remote.empty()) return fail(h, PK_E_UNSUPPORTED, "the unsplit scheme runs on one rank");
        if (int rc = exchange_prepare(h)) return rc;
    }
    for (auto& b : h->blocks) {
        if (!h->connected && !b.uh) PK_CUDA(h, cudaMalloc(&b.uh, sizeof(double) * h->nplanes * b.plane));
        for (int d = 0; d < 3; ++d)
            if (b.n[d] > 1 && !b.flux[d]) PK_CUDA(h, cudaMalloc(&b.flux[d], sizeof(double) * h->nplanes * b.plane));
    }
    for (int s = 1; s <= nst; ++s) {
        const bool first = s == 1;
        const int last = (order == 1) || (s == 2);
        const double rk = order == 1 ? 1.0 : (first ? 0.5 : 1.0);
        const bool to_uh = order == 2 && first;
        // the face fluxes, finest level first: a refined block's fluxes through
        // faces bordering the coarser level are restricted into that level's
        // flux through the same face before its blocks compute theirs
        // (unsplit_sweeps.F90:132-177 with fc_fluxes_unsplit.F90)
        for (int L = h->max_level; L >= 0; --L) {
            for (auto& b : h->blocks) {
                if (b.level != L) continue;
                double* u = state(h, b);
                double* uh = h->connected ? b.buf[1 - h->cur] : b.uh;
                const double* in = (first || order < 2) ? u : uh;
                for (int d = 0; d < 3; ++d)
                    if (b.n[d] > 1)
                        if (int rc = ops->unsplit_flux(h, b, d, in, b.flux[d])) return rc;
            }
            if (L > 0)
                for (int d = 0; d < 3; ++d) {
                    if (!h->d_src[d]) continue;
                    const int beg = h->in_level_beg[d][L - 1], end = h->in_level_beg[d][L];
                    if (end <= beg) continue;
                    const long long n = (long long)(end - beg) * h->nplanes;
                    k_restrict_flux<<<grid1d(n, 256), 256, 0, h->stream>>>(h->d_src[d], beg, end, h->nplanes,
                                                                           h->d_out_flux[d], h->d_in_flux[d],
                                                                           h->fc_scale);
                    PK_CUDA(h, cudaGetLastError());
                    h->launches += 1;
                }
        }
        for (auto& b : h->blocks) {
            double* u = state(h, b);
            double* uh = h->connected ? b.buf[1 - h->cur] : b.uh;
            double* T = to_uh ? uh : u;
            if (int rc = ops->unsplit_apply(h, b, u, T, rk, last)) return rc;
            if (h->max_level == 0)                     // refined domains overwrite every guard cell below
                if (int rc = fill_guards_ptr(h, b, T)) return rc;
            b.guards_stale = false;
        }
        // update_boundaries(istep) between the blocks (unsplit_sweeps.F90:182):
        // same-level copies, then prolongation coarsest level first
        if (h->connected) {
            const int par = to_uh ? 1 - h->cur : h->cur;
            if (h->xlocal.total > 0) {
                const int nblk = (int)(h->xlocal.n < grid_cap() ? h->xlocal.n : grid_cap());
                k_exchange<<<nblk, 256, 0, h->stream>>>(h->xlocal.dev, h->xlocal.n, h->xlocal.total, h->d_xptr[par],
                                                        h->nplanes);
                PK_CUDA(h, cudaGetLastError());
                h->launches += 1;
            }
            if (h->max_level > 0)
                if (int rc = prolong_guards(h, -1, par)) return rc;
        }
    }
    return PK_OK;
}

// fluid_update_unsplit (unsplit_fluidupdate.F90:45-126)
static int unsplit_fluid_update(pk_ctx* h)
{
    const double dt = h->ts.dt;
    double ch = h->ts.chspeed, fac = 1.0;
    if (h->cfg.magnetic) {
        double fac_full;
        if (int rc = glm_scalars_for(h, dt, h->ts.chspeed, &ch, &fac_full)) return rc;   // update_chspeed
        fac = glm_fac_for(h, dt / 2.0, ch);                      // glmdamping(half = .true.): dt_eff = dt/2
        h->ts.chspeed = ch;
    }
    if (int rc = put_step_params(h, dt, ch, fac)) return rc;
    if (h->cfg.magnetic)
        if (int rc = glm_scale(h, fac)) return rc;
    h->ts.t = h->ts.t + dt;                           // unsplit_fluidupdate.F90:98
    if (int rc = unsplit_sweep(h)) return rc;
    if (h->cfg.magnetic)
        if (int rc = glm_scale(h, fac)) return rc;
    return PK_OK;
}

// time_step of every stacked instance: its own CFL reduction and clamps
static int inst_time_step(pk_ctx* h)
{
    Block& b = h->blocks[0];
    const int ni = h->ninst;
    if (ni > h->red_cap / 12) return fail(h, PK_E_STATE, "reduction slots too few for the instances");
    PK_CUDA(h, cudaMemsetAsync(h->d_red, 0, sizeof(unsigned long long) * 12 * ni, h->stream));
    CflArgs a;
    a.nfl = h->cfg.nfluids;
    int beg = 0;
    for (int f = 0; f < 3; ++f) {
        a.fl[f].kind = f < a.nfl ? h->cfg.fluid_kind[f] : K_NONE;
        a.fl[f].beg = beg;
        a.fl[f].gam = h->pp.gam[f];
        a.fl[f].gam_1 = h->pp.gam_1[f];
        if (f < a.nfl) beg += (h->cfg.fluid_kind[f] == PK_FLUID_DST) ? 4 : 5;
    }
    a.magnetic = h->cfg.magnetic;
    a.ib = h->ib;
    k_cfl_blocks<<<dim3(64, ni), 256, 0, h->stream>>>(h->d_inst[h->cur], a, h->d_red);
    PK_CUDA(h, cudaGetLastError());
    h->launches += 1;
    PK_CUDA(h, cudaMemcpyAsync(h->h_red, h->d_red, sizeof(unsigned long long) * 12 * ni, cudaMemcpyDeviceToHost,
                               h->stream));
    PK_CUDA(h, cudaStreamSynchronize(h->stream));
    for (int i = 0; i < ni; ++i) {
        double dt = DBL_MAX, c_all = 0.0;
        for (int f = 0; f < h->cfg.nfluids; ++f) {
            double cm[4];
            for (int d = 0; d < 4; ++d) std::memcpy(&cm[d], &h->h_red[12 * i + 4 * f + d], sizeof(double));
            double dtp[3];
            for (int d = 0; d < 3; ++d) dtp[d] = (b.n[d] > 1 && cm[d] > 0.0) ? b.dl[d] / cm[d] : DBL_MAX;
            double m = dtp[0];
            m = (dtp[1] < m) ? dtp[1] : m;
            m = (dtp[2] < m) ? dtp[2] : m;
            const double dtf = h->cfg.cfl * m;
            dt = (dtf < dt) ? dtf : dt;
            c_all = (cm[3] > c_all) ? cm[3] : c_all;
        }
        pk_time_state& ts = h->its[i];
        ts.dt_old = ts.dt;
        if (clamp_dt(h->cfg, ts, dt, c_all)) return fail(h, PK_E_DTMIN, "dt < dt_min in an instance");
    }
    h->ts = h->its[0];
    return PK_OK;
}

// fluid_update_full of every stacked instance with its own dt (one launch per sweep)
static int inst_fluid_update(pk_ctx* h, std::vector<StepRec>* record)
{
    const int ni = h->ninst;
    std::vector<StepRec> r(ni);
    for (int i = 0; i < ni; ++i) {
        pk_time_state& ts = h->its[i];
        double ch, fac;
        if (int rc = glm_scalars_for(h, ts.dt, ts.chspeed, &ch, &fac)) return rc;
        ts.chspeed = ch;
        r[i] = StepRec{ts.dt, ch, fac};
    }
    if (int rc = put_step_array(h, r.data())) return rc;
    if (int rc = run_step_sweeps(h, r[0].dt, r[0].ch, r[0].fac)) return rc;
    for (int i = 0; i < ni; ++i) {
        pk_time_state& ts = h->its[i];
        ts.t = ts.t + ts.dt;                          // fluidupdate.F90:116, :126
        ts.t = ts.t + ts.dt;
    }
    if (record) record->insert(record->end(), r.begin(), r.end());
    h->ts = h->its[0];
    return PK_OK;
}

int pk_time_step(pk_handle h, double* dt_out)
{
    if (!h) return PK_E_ARG;
    if (h->ninst > 1) {
        const int rc = inst_time_step(h);
        if (dt_out) *dt_out = h->its[0].dt;
        return rc;
    }
    double dt, c_all;
    h->ts.dt_old = h->ts.dt;                          // timestep.F90:158
    if (int rc = pk_timestep_raw(h, &dt, &c_all)) return rc;
    if (h->reduce_cb) {                               // over ranks (timestep.F90:173, MPI_MIN / MPI_MAX)
        dt = h->reduce_cb(h->comm_ctx, dt, 0);
        c_all = h->reduce_cb(h->comm_ctx, c_all, 1);
    }
    const int rc = clamp_dt(h->cfg, h->ts, dt, c_all);
    if (dt_out) *dt_out = h->ts.dt;
    if (rc) return fail(h, PK_E_DTMIN, "dt < dt_min");
    return PK_OK;
}

int pk_fluid_update(pk_handle h)
{
    if (!h) return PK_E_ARG;
    if (h->blocks.empty()) return fail(h, PK_E_STATE, "no block registered");
    if (h->cfg.solver == PK_SOLVER_UNSPLIT) return unsplit_fluid_update(h);
    if (h->ninst > 1) return inst_fluid_update(h, nullptr);
    const double dt = h->ts.dt;
    double ch, fac;
    if (int rc = glm_scalars(h, dt, &ch, &fac)) return rc;
    h->ts.chspeed = ch;
    if (int rc = put_step_params(h, dt, ch, fac)) return rc;
    if (int rc = run_step_sweeps(h, dt, ch, fac)) return rc;
    h->ts.t = h->ts.t + dt;                            // fluidupdate.F90:116
    h->ts.t = h->ts.t + dt;                            // :126
    return PK_OK;
}

// cfl_max after the sanitising of init_global (global.F90:304)
static double cfl_max_of(const pk_config& c)
{
    const double x = c.cfl;
    double lo = (x * 1.1 < x + 0.05) ? x * 1.1 : x + 0.05;
    lo = ((1.0 + x) / 2.0 < lo) ? (1.0 + x) / 2.0 : lo;
    const double m = (lo > c.cfl_max) ? lo : c.cfl_max;
    return (1.0 < m) ? 1.0 : m;
}

// dt_shrink**n as an integer power: repeated squaring
static double powi(double x, int n)
{
    double r = 1.0;
    while (n > 0) {
        if (n & 1) r = r * x;
        x = x * x;
        n >>= 1;
    }
    return r;
}

// stepcfl of cfl_warn (timestep.F90:329-330)
static double stepcfl_of(const pk_ctx* h, double c_all_old, double c_all)
{
    double s = h->cfg.cfl * h->ts.dt_cur_shrink;
    if (c_all_old > 0.0) s = ((c_all / c_all_old) * h->cfg.cfl) * h->ts.dt_cur_shrink;
    return s;
}

// the state copy of repeat_fluidstep: save (restore = 0) or restore (1)
static int retry_copy(pk_ctx* h, int restore)
{
    for (auto& b : h->blocks) {
        const size_t bytes = sizeof(double) * h->nplanes * b.plane;
        if (!b.retry) {
            if (cudaMalloc(&b.retry, bytes) != cudaSuccess) return fail(h, PK_E_NOMEM, "cudaMalloc of the retry copy failed");
        }
        if (b.guards_stale && !restore)
            if (int rc = refresh_guards(h, b)) return rc;
        if (restore) PK_CUDA(h, cudaMemcpyAsync(state(h, b), b.retry, bytes, cudaMemcpyDeviceToDevice, h->stream));
        else PK_CUDA(h, cudaMemcpyAsync(b.retry, state(h, b), bytes, cudaMemcpyDeviceToDevice, h->stream));
        if (restore) b.guards_stale = false;
    }
    return PK_OK;
}

// check_cfl_violation (timestep.F90:247-310) with cfl_warn from the
// non-main time_step call: sets repeat_step and dt_cur_shrink
static int check_cfl(pk_ctx* h)
{
    uint32_t st = 0;
    if (int rc = pk_status(h, &st)) return rc;
    double neg = (st & (PK_ST_DN_NEGATIVE | PK_ST_EI_NEGATIVE)) ? 1.0 : 0.0;
    if (h->reduce_cb) neg = h->reduce_cb(h->comm_ctx, neg, 1);        // pLOR
    const int unwanted = (neg > 0.0 && h->cfg.disallow_negatives) ? 1 : 0;
    double dt, c_all;                                                // time_step(checkdt, flind, .false.)
    if (int rc = pk_timestep_raw(h, &dt, &c_all)) return rc;
    if (h->reduce_cb) {
        dt = h->reduce_cb(h->comm_ctx, dt, 0);
        c_all = h->reduce_cb(h->comm_ctx, c_all, 1);
    }
    const pk_config& c = h->cfg;
    if (h->ts.nstep < 1) {
        if (c.dt_initial > 0.0) dt = (c.dt_initial < dt) ? c.dt_initial : dt;
        else if (c.dt_initial < 0.0) {
            const double x = -c.dt_initial * dt;
            dt = (x < dt) ? x : dt;
        }
    } else if (h->ts.dt_old > 0.0) {
        const double x = h->ts.dt_old * c.dt_max_grow;
        dt = (x < dt) ? x : dt;
    }
    h->ts.stepcfl = stepcfl_of(h, h->ts.c_all_old, c_all);
    int repeat = unwanted;
    if (h->ts.stepcfl > cfl_max_of(c)) repeat = 1;
    if (!repeat) {
        h->ts.dt_cur_shrink = 1.0;
    } else if (c.cflcontrol == PK_CFL_FLEX) {          // flexible_shrink (timestep.F90:347-349)
        h->ts.dt_cur_shrink = cfl_max_of(c) / h->ts.stepcfl;
        if (h->ts.tstep_attempt >= 1) h->ts.dt_cur_shrink = h->ts.dt_cur_shrink * c.dt_shrink;
    } else {
        h->ts.dt_cur_shrink = powi(c.dt_shrink, h->ts.tstep_attempt + 1);
    }
    if (dt < c.dt_min) return fail(h, PK_E_DTMIN, "dt < dt_min in the check after the step");
    h->ts.repeat_step = repeat;
    return PK_OK;
}

// piernik.F90:125-167: the main loop body nsteps times (a redone step counts
// as one), with the retry machinery when cflcontrol = redo
int pk_run(pk_handle h, int32_t nsteps)
{
    if (!h) return PK_E_ARG;
    if (h->ninst > 1) {                                // stacked instances: each its own dt
        for (int s = 0; s < nsteps; ++s) {
            if (int rc = inst_time_step(h)) return rc;
            if (int rc = inst_fluid_update(h, nullptr)) return rc;
            for (auto& ts : h->its) ts.nstep += 1;
            h->ts = h->its[0];
        }
        return PK_OK;
    }
    const int redo = h->cfg.cflcontrol == PK_CFL_REDO || h->cfg.cflcontrol == PK_CFL_FLEX;   // repetitive_steps
    for (int s = 0; s < nsteps; ++s) {
        if (!(h->ts.t < h->cfg.tend) && !h->ts.repeat_step) break;
        if (!h->ts.repeat_step) {
            const double c_old = h->ts.c_all_old;
            const int rc = pk_time_step(h, nullptr);
            if (h->cfg.cflcontrol == PK_CFL_WARN) h->ts.stepcfl = stepcfl_of(h, c_old, h->ts.c_all);
            h->ts.c_all_old = h->ts.c_all;
            if (rc) return rc;
            h->ts.dt_full = h->ts.dt;
        }
        if (redo) {                                      // repeat_fluidstep
            if (h->ts.repeat_step) {
                h->ts.tstep_attempt += 1;
                if (h->ts.tstep_attempt > h->cfg.max_redostep_attempts)
                    return fail(h, PK_E_STATE, "tstep_attempt > max_redostep_attempts");
                h->ts.t = h->ts.t_saved;
                h->ts.nstep = h->ts.nstep_saved;
                h->ts.dt = h->ts.dt_full * h->ts.dt_cur_shrink;
                if (int rc = retry_copy(h, 1)) return rc;
                h->ts.redone += 1;
            } else {
                h->ts.tstep_attempt = 0;
                h->ts.nstep_saved = h->ts.nstep;
                h->ts.t_saved = h->ts.t;
                if (int rc = retry_copy(h, 0)) return rc;
            }
        }
        if (int rc = pk_fluid_update(h)) return rc;
        h->ts.nstep += 1;
        if (redo)
            if (int rc = check_cfl(h)) return rc;
    }
    return PK_OK;
}

int pk_get_time_state(pk_handle h, pk_time_state* st)
{
    if (!h || !st) return PK_E_ARG;
    *st = h->ts;
    return PK_OK;
}

int pk_set_time_state(pk_handle h, const pk_time_state* st)
{
    if (!h || !st) return PK_E_ARG;
    h->ts = *st;
    if (h->ninst > 1) h->its.assign(h->ninst, *st);   // stacked instances: every one
    return PK_OK;
}

int pk_status(pk_handle h, uint32_t* flags)
{
    if (!h || !flags) return PK_E_ARG;
    unsigned s = 0;
    PK_CUDA(h, cudaMemcpyAsync(&s, h->d_status, sizeof(unsigned), cudaMemcpyDeviceToHost, h->stream));
    PK_CUDA(h, cudaMemsetAsync(h->d_status, 0, sizeof(unsigned), h->stream));
    PK_CUDA(h, cudaStreamSynchronize(h->stream));
    *flags = s;
    return PK_OK;
}

int pk_sync(pk_handle h)
{
    if (!h) return PK_E_ARG;
    PK_CUDA(h, cudaStreamSynchronize(h->stream));
    return PK_OK;
}

int pk_set_arithmetic(pk_handle h, int32_t mode)
{
    if (!h) return PK_E_ARG;
    if (mode != PK_ARITH_BITEXACT && mode != PK_ARITH_FMA) return fail(h, PK_E_ARG, "unknown arithmetic mode");
    if (mode == PK_ARITH_FMA)
        if (int rc = fast_ops_of(h)->prepare(h)) return rc;   // kernel attributes, before any capture
    if (mode != h->arith) invalidate_graph(h);
    h->arith = mode;
    return PK_OK;
}

int pk_set_tile(pk_handle h, int32_t dir, int32_t pencils, int32_t length, int32_t variant)
{
    if (!h || dir < 0 || dir > 2 || pencils < 0 || length < 0 || variant < -1 || variant >= NVARIANT) return PK_E_ARG;
    const int maxt = VAR_T[variant >= 0 ? variant : 0];
    // a length of a whole periodic pencil runs without halo (up to the CTA size);
    // any other length needs its 8 halo cells inside the CTA (checked at launch)
    if (length > maxt) return fail(h, PK_E_ARG, "length exceeds the variant's CTA size");
    h->tileP[dir] = pencils;
    h->tileL[dir] = length;
    h->tileV[dir] = variant;
    invalidate_graph(h);
    return PK_OK;
}

int pk_set_batch(pk_handle h, int32_t enable, int32_t length, int32_t variant)
{
    if (!h || length < 0 || variant < -1 || variant >= NVARIANT) return PK_E_ARG;
    const int v = variant >= 0 ? variant : h->batch_variant;
    const int L = length > 0 ? length : h->batch_L;
    if (L + 8 > VAR_T[v]) return fail(h, PK_E_ARG, "length + 8 exceeds the variant's CTA size");
    h->batched = enable != 0;
    h->batch_variant = v;
    h->batch_L = L;
    h->batch_dirty = true;
    invalidate_graph(h);
    return PK_OK;
}

int pk_set_refined_launch(pk_handle h, int32_t one_launch)
{
    if (!h) return PK_E_ARG;
    h->refined_one_launch = one_launch != 0;
    invalidate_graph(h);
    return PK_OK;
}

int pk_use_graph(pk_handle h, int32_t enable)
{
    if (!h) return PK_E_ARG;
    h->use_graph = enable != 0;
    invalidate_graph(h);
    return PK_OK;
}

int pk_tile_variants(int32_t* n, int32_t* threads, int32_t* ctas_per_sm)
{
    if (n) *n = NVARIANT;
    for (int v = 0; v < NVARIANT; ++v) {
        if (threads) threads[v] = VAR_T[v];
        if (ctas_per_sm) ctas_per_sm[v] = VAR_B[v];
    }
    return PK_OK;
}

int pk_profile_enable(pk_handle h, int32_t on)
{
    if (!h) return PK_E_ARG;
    h->profiling = on != 0;
    return PK_OK;
}

int pk_profile_read(pk_handle h, int64_t* launches, int64_t* sweep_launches, double* sweep_ms)
{
    if (!h) return PK_E_ARG;
    PK_CUDA(h, cudaStreamSynchronize(h->stream));
    double ms = 0.0;
    for (auto& p : h->ev_used) {
        float x = 0.0f;
        PK_CUDA(h, cudaEventElapsedTime(&x, p.first, p.second));
        ms += x;
        h->ev_free.push_back(p);
    }
    const long long timed = (long long)h->ev_used.size();
    h->ev_used.clear();
    if (launches) *launches = h->launches;
    if (sweep_launches) *sweep_launches = timed;
    if (sweep_ms) *sweep_ms = ms;
    return PK_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Differentiable path: recorded forward with checkpoints, adjoint backward
// ---------------------------------------------------------------------------

namespace {

void grad_release(pk_ctx* h)
{
    cudaStreamSynchronize(h->stream);
    for (double* p : h->grad_ckpt) cudaFree(p);
    for (double* p : h->grad_pool) cudaFree(p);
    for (double* p : h->grad_star) cudaFree(p);
    for (unsigned short* p : h->grad_flags) cudaFree(p);
    h->grad_ckpt.clear();
    h->grad_pool.clear();
    h->grad_star.clear();
    h->grad_flags.clear();
    h->grad_steps.clear();
}

int grad_check(pk_ctx* h)
{
    if (h->blocks.size() != 1 || !h->remote.empty())
        return fail(h, PK_E_UNSUPPORTED, "the differentiable path runs on one block of one rank");
    if (!fused_ok(h)) return fail(h, PK_E_UNSUPPORTED, "the differentiable path needs RK2 and periodic boundaries");
    if (h->cfg.nfluids != 1) return fail(h, PK_E_UNSUPPORTED, "the differentiable path is built for one fluid");
    if (h->cfg.use_eglm) return fail(h, PK_E_UNSUPPORTED, "the differentiable path has no E-GLM sources");
    if (h->cfg.interpolation != PK_INTERP_LINEAR)
        return fail(h, PK_E_UNSUPPORTED, "the differentiable path differentiates the linear (limited) reconstruction");
    int dirs[3], nd;
    step_dirs(h, dirs, &nd);
    if (nd == 0) return fail(h, PK_E_UNSUPPORTED, "the differentiable path needs at least one swept direction");
    return ensure_pingpong(h);
}

int alloc_state(pk_ctx* h, const Block& b, double** p)
{
    if (cudaMalloc(p, sizeof(double) * h->nplanes * b.plane) != cudaSuccess)
        return fail(h, PK_E_NOMEM, "cudaMalloc for the differentiable path failed");
    PK_CUDA(h, cudaMemsetAsync(*p, 0, sizeof(double) * h->nplanes * b.plane, h->stream));
    return PK_OK;
}

// room for the recomputed sweeps of `need` sweeps (output, stage-1 state,
// floor records) and the adjoint sweep's scratch state
int ensure_pool(pk_ctx* h, const Block& b, int need)
{
    while ((int)h->grad_pool.size() < need) {
        double *p, *q;
        if (int rc = alloc_state(h, b, &p)) return rc;
        h->grad_pool.push_back(p);
        if (int rc = alloc_state(h, b, &q)) return rc;
        h->grad_star.push_back(q);
        unsigned short* f;
        if (cudaMalloc(&f, sizeof(unsigned short) * b.plane) != cudaSuccess)
            return fail(h, PK_E_NOMEM, "cudaMalloc for the differentiable path failed");
        h->grad_flags.push_back(f);
    }
    if (!h->lam_m1)
        if (int rc = alloc_state(h, b, &h->lam_m1)) return rc;
    return PK_OK;
}

// the sweeps of one step as (direction, damping applied) pairs, in step_sweeps' order
int step_plan(pk_ctx* h, int* dir, int* fac)
{
    int dirs[3], nd;
    step_dirs(h, dirs, &nd);
    int k = 0;
    for (int half = 0; half < 2; ++half)
        for (int s = 0; s < nd; ++s) {
            dir[k] = half == 0 ? dirs[s] : dirs[nd - 1 - s];
            fac[k] = h->cfg.magnetic && s == nd - 1;
            ++k;
        }
    return k;
}

}  // namespace

extern "C" {

int pk_upload_device(pk_handle h, int32_t id, const double* soa_dev)
{
    Block* b;
    if (int rc = get_block(h, id, &b)) return rc;
    if (!soa_dev) return fail(h, PK_E_ARG, "null array");
    PK_CUDA(h, cudaMemcpyAsync(state(h, *b), soa_dev, sizeof(double) * h->nplanes * b->plane, cudaMemcpyDeviceToDevice,
                               h->stream));
    return fill_guards_block(h, *b);
}

int pk_download_device(pk_handle h, int32_t id, double* soa_dev)
{
    Block* b;
    if (int rc = get_block(h, id, &b)) return rc;
    if (!soa_dev) return fail(h, PK_E_ARG, "null array");
    if (b->guards_stale)
        if (int rc = refresh_guards(h, *b)) return rc;
    PK_CUDA(h, cudaMemcpyAsync(soa_dev, state(h, *b), sizeof(double) * h->nplanes * b->plane, cudaMemcpyDeviceToDevice,
                               h->stream));
    PK_CUDA(h, cudaStreamSynchronize(h->stream));
    return PK_OK;
}

int pk_adjoint_set(pk_handle h, int32_t id, const double* lam, int32_t on_device)
{
    Block* b;
    if (int rc = get_block(h, id, &b)) return rc;
    if (!lam) return fail(h, PK_E_ARG, "null array");
    if (!h->lam)
        if (int rc = alloc_state(h, *b, &h->lam)) return rc;
    if (!h->lam_tmp)
        if (int rc = alloc_state(h, *b, &h->lam_tmp)) return rc;
    PK_CUDA(h, cudaMemcpyAsync(h->lam, lam, sizeof(double) * h->nplanes * b->plane,
                               on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, h->stream));
    // the sweeps read periodic images of the interior only: guard values carry no derivative
    k_zero_guards<<<grid1d(b->plane, 256), 256, 0, h->stream>>>(box_of(*b), h->lam, h->nplanes);
    PK_CUDA(h, cudaGetLastError());
    h->launches += 1;
    PK_CUDA(h, cudaStreamSynchronize(h->stream));
    return PK_OK;
}

int pk_adjoint_get(pk_handle h, int32_t id, double* lam, int32_t on_device)
{
    Block* b;
    if (int rc = get_block(h, id, &b)) return rc;
    if (!lam || !h->lam) return fail(h, PK_E_STATE, "no adjoint state");
    PK_CUDA(h, cudaMemcpyAsync(lam, h->lam, sizeof(double) * h->nplanes * b->plane,
                               on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, h->stream));
    PK_CUDA(h, cudaStreamSynchronize(h->stream));
    return PK_OK;
}

int pk_adjoint_sweep(pk_handle h, int32_t cdim, double dt, double chspeed)
{
    if (!h) return PK_E_ARG;
    if (cdim < 1 || cdim > 3) return fail(h, PK_E_ARG, "cdim must be 1..3");
    if (int rc = grad_check(h)) return rc;
    if (!h->lam) return fail(h, PK_E_STATE, "set the adjoint first (pk_adjoint_set)");
    Block& b = h->blocks[0];
    const PhysOps* ops = ops_of(h);
    if (int rc = ensure_pool(h, b, 1)) return rc;
    if (int rc = put_step_params(h, dt, chspeed, 1.0)) return rc;
    const int d = cdim - 1;
    if (int rc = ops->fused_rec(h, b, d, 0, state(h, b), h->grad_pool[0], h->grad_star[0], h->grad_flags[0])) return rc;
    if (int rc = ops->adj(h, b, d, 0, state(h, b), h->grad_star[0], h->grad_pool[0], h->grad_flags[0], h->lam,
                          h->lam_tmp, h->lam_m1))
        return rc;
    std::swap(h->lam, h->lam_tmp);
    PK_CUDA(h, cudaStreamSynchronize(h->stream));
    return PK_OK;
}

int pk_grad_forward(pk_handle h, int32_t nsteps, int32_t every, const double* dt_in, double* dt_out)
{
    if (!h || nsteps < 0 || every < 1) return PK_E_ARG;
    if (int rc = grad_check(h)) return rc;
    Block& b = h->blocks[0];
    h->grad_steps.clear();                            // checkpoint buffers of an earlier recording are reused
    h->grad_every = every;
    h->grad_ts0 = h->ts;
    for (int s = 0; s < nsteps; ++s) {
        if (s % every == 0) {
            const size_t k = (size_t)(s / every);
            if (k >= h->grad_ckpt.size()) {
                double* p;
                if (int rc = alloc_state(h, b, &p)) return rc;
                h->grad_ckpt.push_back(p);
            }
            PK_CUDA(h, cudaMemcpyAsync(h->grad_ckpt[k], state(h, b), sizeof(double) * h->nplanes * b.plane,
                                       cudaMemcpyDeviceToDevice, h->stream));
        }
        if (h->ninst > 1) {                            // stacked instances: ninst step records per step
            const int ni = h->ninst;
            if (dt_in) {
                for (int i = 0; i < ni; ++i) {
                    h->its[i].dt_old = h->its[i].dt;
                    h->its[i].dt = dt_in[(size_t)s * ni + i];
                }
            } else {
                if (int rc = inst_time_step(h)) return rc;
            }
            if (int rc = inst_fluid_update(h, &h->grad_steps)) return rc;
            for (auto& ts : h->its) ts.nstep += 1;
            h->ts = h->its[0];
            if (dt_out)
                for (int i = 0; i < ni; ++i) dt_out[(size_t)s * ni + i] = h->its[i].dt;
            continue;
        }
        double dt;
        if (dt_in) {
            h->ts.dt_old = h->ts.dt;
            dt = dt_in[s];
            h->ts.dt = dt;
        } else {
            if (int rc = pk_time_step(h, &dt)) return rc;
        }
        double ch, fac;
        if (int rc = glm_scalars(h, dt, &ch, &fac)) return rc;
        h->ts.chspeed = ch;
        if (int rc = put_step_params(h, dt, ch, fac)) return rc;
        if (int rc = step_sweeps(h, dt, ch, fac)) return rc;
        h->ts.t = h->ts.t + dt;                        // two half steps of dt, as pk_fluid_update
        h->ts.t = h->ts.t + dt;
        h->ts.nstep += 1;
        h->grad_steps.push_back(StepRec{dt, ch, fac});
        if (dt_out) dt_out[s] = dt;
    }
    PK_CUDA(h, cudaStreamSynchronize(h->stream));
    return PK_OK;
}

int pk_grad_backward(pk_handle h)
{
    if (!h) return PK_E_ARG;
    if (int rc = grad_check(h)) return rc;
    if (!h->lam) return fail(h, PK_E_STATE, "set the adjoint of the final state first (pk_adjoint_set)");
    Block& b = h->blocks[0];
    const PhysOps* ops = ops_of(h);
    int dir[6], fac[6];
    const int nsw = step_plan(h, dir, fac);
    const int ni = h->ninst;
    const int K = (int)h->grad_steps.size() / ni, C = h->grad_every;
    if (K == 0) return PK_OK;
    if (int rc = ensure_pool(h, b, C * nsw)) return rc;
    const int nseg = (K + C - 1) / C;
    for (int seg = nseg - 1; seg >= 0; --seg) {
        const int s0 = seg * C, len = (K - s0 < C) ? K - s0 : C;
        // recompute the segment, keeping every sweep's output
        const double* x = h->grad_ckpt[seg];
        for (int j = 0; j < len; ++j) {
            if (int rc = put_step_array(h, &h->grad_steps[(size_t)(s0 + j) * ni])) return rc;
            for (int k = 0; k < nsw; ++k) {
                const int i = j * nsw + k;
                if (int rc = ops->fused_rec(h, b, dir[k], fac[k], x, h->grad_pool[i], h->grad_star[i], h->grad_flags[i]))
                    return rc;
                x = h->grad_pool[i];
            }
        }
        // adjoint sweeps back to the segment's start
        for (int j = len - 1; j >= 0; --j) {
            if (int rc = put_step_array(h, &h->grad_steps[(size_t)(s0 + j) * ni])) return rc;
            for (int k = nsw - 1; k >= 0; --k) {
                const int i = j * nsw + k;
                const double* uin = i > 0 ? h->grad_pool[i - 1] : h->grad_ckpt[seg];
                if (int rc = ops->adj(h, b, dir[k], fac[k], uin, h->grad_star[i], h->grad_pool[i], h->grad_flags[i],
                                      h->lam, h->lam_tmp, h->lam_m1))
                    return rc;
                std::swap(h->lam, h->lam_tmp);
            }
        }
    }
    PK_CUDA(h, cudaStreamSynchronize(h->stream));
    return PK_OK;
}

int pk_restrict(pk_handle h)
{
    if (!h) return PK_E_ARG;
    if (int rc = exchange_prepare(h)) return rc;
    for (int L = h->max_level; L >= 1; --L) {         // restrict_to_base: finest level first
        const long long cells = h->rbox_cells[L];
        if (!cells) continue;
        const int r0 = h->rbox_beg[L], nr = h->rbox_beg[L + 1] - r0;
        k_restrict<<<grid1d(cells, 256), 256, 0, h->stream>>>(h->d_rbox + r0, h->d_rbox_start + r0, nr, cells,
                                                               h->d_xptr[h->cur], h->nplanes, h->dom[0] > 1,
                                                               h->dom[1] > 1, h->dom[2] > 1,
                                                               1.0 / std::ldexp(1.0, h->eff_dim));
        PK_CUDA(h, cudaGetLastError());
        h->launches += 1;
    }
    PK_CUDA(h, cudaStreamSynchronize(h->stream));
    return PK_OK;
}

int pk_prolong_block(pk_handle h, int32_t id)
{
    Block* b;
    if (int rc = get_block(h, id, &b)) return rc;
    if (int rc = exchange_prepare(h)) return rc;
    if (h->max_level < 1 || b->level < 1) return fail(h, PK_E_ARG, "only a block of a refined level can be prolonged");
    const int nl = (int)h->blocks.size();
    std::vector<LBlock> lb(nl);
    for (int i = 0; i < nl; ++i) {
        const Block& x = h->blocks[i];
        lb[i].level = x.level;
        for (int d = 0; d < 3; ++d) {
            lb[i].n[d] = x.n[d];
            lb[i].g[d] = x.g[d];
            lb[i].off[d] = x.off[d];
        }
    }
    std::vector<PRun> runs;
    std::string err;
    if (!build_fill_runs(lb, h->dom, id, runs, err)) return fail(h, PK_E_ARG, err);
    std::vector<PRunDev> dev(runs.size());
    std::vector<long long> start(runs.size());
    long long total = 0;
    for (size_t r = 0; r < runs.size(); ++r) {
        const PRun& s = runs[r];
        dev[r] = PRunDev{s.fb, s.cb, s.fx, s.fy, s.fz, s.len, s.cx, s.cy, s.cz, s.px, s.py, s.pz};
        start[r] = total;
        total += s.len;
    }
    PRunDev* d_runs = nullptr;
    long long* d_start = nullptr;
    int rc = upload_vec(h, dev, &d_runs);
    if (rc == PK_OK) rc = upload_vec(h, start, &d_start);
    // u and B are rank-4 arrays, prolonged by injection whatever their order
    // (cg_level_connected.F90:1063, the QUIRKY ord_prolong = 0); psi with its
    // own order, ord_mag_prolong
    ProlongCoef inj{};
    prolong_coef(0, &inj);
    if (rc == PK_OK && total > 0) {
        k_prolong<<<grid1d(total, 256), 256, 0, h->stream>>>(d_runs, d_start, (int)runs.size(), total,
                                                             h->d_xptr[h->cur], h->nvf, h->cfg.magnetic ? 4 : 0,
                                                             h->dom[0] > 1, h->dom[1] > 1, h->dom[2] > 1, inj, inj,
                                                             h->pro_b);
        if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(h->stream) != cudaSuccess)
            rc = fail(h, PK_E_CUDA, "prolongation of a block failed");
        h->launches += 1;
    }
    cudaFree(d_runs);
    cudaFree(d_start);
    return rc;
}

int pk_mark_refinement(pk_handle h, const pk_urc* crit, int32_t ncrit, int32_t* flagged)
{
    if (!h || (ncrit > 0 && !crit) || ncrit < 0) return PK_E_ARG;
    if (h->ninst > 1) return fail(h, PK_E_STATE, "stacked instances are not refined");
    std::vector<UrcDev> cr(ncrit);
    for (int c = 0; c < ncrit; ++c) {
        if (crit[c].method < PK_URC_THRESHOLD || crit[c].method > PK_URC_LOECHNER)
            return fail(h, PK_E_ARG, "unknown refinement criterion");
        if (crit[c].field < 0 || crit[c].field >= h->nplanes) return fail(h, PK_E_ARG, "criterion field out of range");
        cr[c] = UrcDev{crit[c].method, crit[c].field, crit[c].thr, crit[c].aux};
        if (crit[c].method == PK_URC_LOECHNER && h->cfg.nb < 4)
            return fail(h, PK_E_ARG, "the Loechner criterion needs nb >= 4");
    }
    if (int rc = pk_fill_guards(h)) return rc;          // all_bnd: up-to-date guard cells
    if (int rc = exchange_prepare(h)) return rc;
    const int nb = (int)h->blocks.size();
    std::vector<MarkBlk> mb;
    std::vector<long long> start;
    std::vector<int> owner;
    long long total = 0;
    for (int i = 0; i < nb; ++i) {
        Block& b = h->blocks[i];
        const long long ncell = b.plane;
        if (!b.flag) PK_CUDA(h, cudaMalloc(&b.flag, ncell));
        PK_CUDA(h, cudaMemsetAsync(b.flag, 0, ncell, h->stream));      // flag%init
        if (b.leaf_cells == 0) continue;                                  // not a leaf block
        MarkBlk m;
        m.u = b.buf[h->cur];
        m.plane = b.plane;
        for (int d = 0; d < 3; ++d) {
            m.ext[d] = b.ext[d];
            m.g[d] = b.g[d];
            m.n[d] = b.n[d];
            m.idl[d] = 1.0 / b.dl[d];
        }
        m.level = b.level;
        m.map = b.flag;
        m.leaf = b.leaf;
        mb.push_back(m);
        start.push_back(total);
        owner.push_back(i);
        total += ncell;
    }
    MarkBlk* d_mb = nullptr;
    long long* d_start = nullptr;
    UrcDev* d_cr = nullptr;
    int* d_flagged = nullptr;
    int rc = upload_vec(h, mb, &d_mb);
    if (rc == PK_OK) rc = upload_vec(h, start, &d_start);
    if (rc == PK_OK) rc = upload_vec(h, cr, &d_cr);
    if (rc == PK_OK && !mb.empty() && cudaMalloc(&d_flagged, sizeof(int) * mb.size()) != cudaSuccess)
        rc = fail(h, PK_E_NOMEM, "cudaMalloc failed");
    std::vector<int> got(mb.size(), 0);
    if (rc == PK_OK && total > 0 && ncrit > 0) {
        cudaMemsetAsync(d_flagged, 0, sizeof(int) * mb.size(), h->stream);
        k_mark<<<grid1d(total, 256), 256, 0, h->stream>>>(d_mb, d_start, (int)mb.size(), total, d_cr, ncrit,
                                                          h->blocks[0].n[0] > 1, h->blocks[0].n[1] > 1,
                                                          h->blocks[0].n[2] > 1, d_flagged);
        h->launches += 1;
        if (cudaGetLastError() != cudaSuccess ||
            cudaMemcpyAsync(got.data(), d_flagged, sizeof(int) * got.size(), cudaMemcpyDeviceToHost, h->stream) !=
                cudaSuccess)
            rc = fail(h, PK_E_CUDA, "refinement marking failed");
    }
    if (rc == PK_OK && cudaStreamSynchronize(h->stream) != cudaSuccess) rc = fail(h, PK_E_CUDA, "refinement marking failed");
    cudaFree(d_mb);
    cudaFree(d_start);
    cudaFree(d_cr);
    cudaFree(d_flagged);
    if (rc == PK_OK && flagged) {
        for (int i = 0; i < nb; ++i) flagged[i] = 0;
        for (size_t k = 0; k < owner.size(); ++k) flagged[owner[k]] = got[k];
    }
    return rc;
}

int pk_refine_map(pk_handle h, int32_t id, uint8_t* map)
{
    Block* b;
    if (int rc = get_block(h, id, &b)) return rc;
    if (!map) return fail(h, PK_E_ARG, "null map");
    if (!b->flag) return fail(h, PK_E_STATE, "no flags: call pk_mark_refinement first");
    PK_CUDA(h, cudaMemcpyAsync(map, b->flag, b->plane, cudaMemcpyDeviceToHost, h->stream));
    PK_CUDA(h, cudaStreamSynchronize(h->stream));
    return PK_OK;
}

int pk_refine_candidates(pk_handle h, int32_t id, const int32_t bsize[3], int64_t* offsets, int32_t cap,
                         int32_t* count)
{
    Block* b;
    if (int rc = get_block(h, id, &b)) return rc;
    if (!bsize || !count || (cap > 0 && !offsets)) return fail(h, PK_E_ARG, "null argument");
    *count = 0;
    std::vector<uint8_t> map((size_t)b->plane);
    if (int rc = pk_refine_map(h, id, map.data())) return rc;
    std::vector<unsigned char> leaf;
    if (b->leaf) {
        leaf.resize((size_t)b->n[0] * b->n[1] * b->n[2]);
        PK_CUDA(h, cudaMemcpy(leaf.data(), b->leaf, leaf.size(), cudaMemcpyDeviceToHost));
    }
    bool has[3];
    long long bs[3], is[3], ie[3];
    for (int d = 0; d < 3; ++d) {
        has[d] = b->n[d] > 1;
        if (has[d] && bsize[d] <= 0) return PK_OK;          // blocky AMR only
        bs[d] = has[d] ? bsize[d] : (1LL << 40);             // huge along directions without extent
        is[d] = b->off[d];
        ie[d] = b->off[d] + b->n[d] - 1;
    }
    // flag%clear(leafmap): drop the flags of covered interior cells
    auto flag_at = [&](long long x, long long y, long long z) -> bool {
        const long long lx = x - b->off[0], ly = y - b->off[1], lz = z - b->off[2];
        const long long c = ((lz + b->g[2]) * b->ext[1] + (ly + b->g[1])) * b->ext[0] + (lx + b->g[0]);
        if (!map[(size_t)c]) return false;
        return leaf.empty() || leaf[(size_t)((lz * b->n[1] + ly) * b->n[0] + lx)];
    };
    const long long rf = 2;
    int found = 0;
    for (long long i = ((is[0]) * rf) / bs[0]; i <= ((ie[0]) * rf + 1) / bs[0]; ++i) {
        const long long ifs = std::max(is[0], (i * bs[0]) / rf), ife = std::min(ie[0], ((i + 1) * bs[0] - 1) / rf);
        for (long long j = ((is[1]) * rf) / bs[1]; j <= ((ie[1]) * rf + 1) / bs[1]; ++j) {
            const long long jfs = std::max(is[1], (j * bs[1]) / rf), jfe = std::min(ie[1], ((j + 1) * bs[1] - 1) / rf);
            for (long long k = ((is[2]) * rf) / bs[2]; k <= ((ie[2]) * rf + 1) / bs[2]; ++k) {
                const long long kfs = std::max(is[2], (k * bs[2]) / rf),
                                kfe = std::min(ie[2], ((k + 1) * bs[2] - 1) / rf);
                bool any = false;
                for (long long z = kfs; z <= kfe && !any; ++z)
                    for (long long y = jfs; y <= jfe && !any; ++y)
                        for (long long x = ifs; x <= ife && !any; ++x) any = flag_at(x, y, z);
                if (!any) continue;
                if (found < cap) {
                    offsets[3 * found + 0] = has[0] ? i * bs[0] : 0;
                    offsets[3 * found + 1] = has[1] ? j * bs[1] : 0;
                    offsets[3 * found + 2] = has[2] ? k * bs[2] : 0;
                }
                ++found;
            }
        }
    }
    *count = found;
    return PK_OK;
}

int pk_set_stage_variant(pk_handle h, int32_t variant)
{
    if (!h) return PK_E_ARG;
    if (variant < 0 || variant >= NSTAGE_VARIANT) return fail(h, PK_E_ARG, "stage variant out of range");
    h->stage_variant = variant;
    h->batch_dirty = true;
    invalidate_graph(h);
    return PK_OK;
}

int pk_set_adjoint_tile(pk_handle h, int32_t dir, int32_t length, int32_t variant)
{
    if (!h) return PK_E_ARG;
    if (dir < -1 || dir > 2 || length < 0 || length > 256 || variant < -1 || variant > 5)
        return fail(h, PK_E_ARG, "adjoint tile: dir -1..2, length 0..256, variant -1..5");
    for (int d = 0; d < 3; ++d)
        if (dir < 0 || dir == d) {
            h->adjL[d] = length;
            h->adjV[d] = variant;
        }
    return PK_OK;
}

int pk_grad_release(pk_handle h)
{
    if (!h) return PK_E_ARG;
    grad_release(h);
    return PK_OK;
}

}  // extern "C"
