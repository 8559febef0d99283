// pk_api.cu -- C ABI of libpiernik_b200.so: block registry, host<->device
// layout conversion, kernel dispatch and the host-side time-step logic of
// PIERNIK's main loop for the split Riemann path.
#include <cuda_runtime.h>

#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/piernik_b200.h"
#include "pk_aux.cuh"
#include "pk_kernels.cuh"

using namespace pk;

namespace {

using PhHD1 = Phys<K_NEU, K_NONE, K_NONE, false>;    // one fluid with energy, no B (solve_cg_u)
using PhMHD1 = Phys<K_ION, K_NONE, K_NONE, true>;    // ionized fluid + B + psi (solve_cg_ub)

enum PhysId { PHYS_HD1 = 0, PHYS_MHD1 = 1 };

constexpr int MAXT = 320;          // threads per CTA of the stage kernel
// Launch-bound variants of the fused sweep (threads per CTA, CTAs per SM): the
// register budget the compiler may use is 65536 / (threads * CTAs); tighter
// budgets trade spills for resident warps.  The autotuner picks per direction.
constexpr int NVARIANT = 6;
constexpr int VAR_T[NVARIANT] = {320, 256, 256, 128, 128, 192};
constexpr int VAR_B[NVARIANT] = {1, 1, 2, 3, 4, 2};
constexpr int DEF_VARIANT[3] = {0, 0, 0};
constexpr int DEF_P[3] = {2, 4, 4};
constexpr int DEF_L[3] = {64, 64, 64};
// ORTHO pairs with the memory-fastest ortho direction first (lanes/coalescing)
constexpr int ORTHO1[3] = {1, 0, 0};
constexpr int ORTHO2[3] = {2, 2, 1};
constexpr int PERM3[3][3] = {{0, 1, 2}, {1, 0, 2}, {2, 1, 0}};

struct Block {
    int n[3], g[3], ext[3];
    double dl[3];
    int bnd[3][2];
    long long plane = 0;
    double* u = nullptr;
    double* uh = nullptr;
    double* tmp = nullptr;
    double* stage = nullptr;   // host-layout conversion buffer
    bool guards_stale = false; // set by the fused sweep, which reads periodic images instead of guards
};

}  // namespace

struct pk_ctx {
    pk_config cfg;
    PhysParams pp;
    int phys = 0;
    int nvf = 0, nplanes = 0, ib = 0;
    std::vector<Block> blocks;
    cudaStream_t stream = nullptr;
    unsigned* d_status = nullptr;
    unsigned long long* d_red = nullptr;
    unsigned long long* h_red = nullptr;
    int red_cap = 0;
    pk_time_state ts;
    std::string err;
    int tileP[3] = {0, 0, 0}, tileL[3] = {0, 0, 0}, tileV[3] = {-1, -1, -1};
    long long launches = 0;          // kernels of this library launched on the handle's stream
    long long sweep_launches = 0;    // of which sweep kernels (fused or stage)
    bool profiling = false;          // bracket sweep kernels with CUDA events
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev_used, ev_free;
};

static int ev_begin(pk_ctx* h, std::pair<cudaEvent_t, cudaEvent_t>* p)
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

static int ev_end(pk_ctx* h, const std::pair<cudaEvent_t, cudaEvent_t>& p)
{
    if (!h->profiling) return PK_OK;
    if (cudaEventRecord(p.second, h->stream) != cudaSuccess) return PK_E_CUDA;
    h->ev_used.push_back(p);
    return PK_OK;
}

#define PK_CUDA(h, call)                                                                      \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess) {                                                              \
            (h)->err = std::string(#call) + ": " + cudaGetErrorString(e_);                   \
            return PK_E_CUDA;                                                                 \
        }                                                                                     \
    } while (0)

static int fail(pk_ctx* h, int code, const std::string& msg)
{
    h->err = msg;
    return code;
}

static int grid1d(long long n, int threads)
{
    long long b = (n + threads - 1) / threads;
    if (b > 148LL * 16) b = 148LL * 16;
    return (int)(b < 1 ? 1 : b);
}

// ---------------------------------------------------------------------------
// kernel launches
// ---------------------------------------------------------------------------

static Geom make_geom(const Block& b, int dir)
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
    return g;
}

template <class PH>
using FusedFn = void (*)(Geom, Tile, const double*, double*, PhysParams, double, double, double, double, unsigned*);

template <class PH>
static FusedFn<PH> fused_variant(int v)
{
    switch (v) {
    case 0: return k_sweep_fused<PH, 320, 1>;
    case 1: return k_sweep_fused<PH, 256, 1>;
    case 2: return k_sweep_fused<PH, 256, 2>;
    case 3: return k_sweep_fused<PH, 128, 3>;
    case 4: return k_sweep_fused<PH, 128, 4>;
    default: return k_sweep_fused<PH, 192, 2>;
    }
}

template <class PH>
static int set_smem_attr(pk_ctx* h)
{
    static bool done = false;
    if (!done) {
        for (int v = 0; v < NVARIANT; ++v)
            PK_CUDA(h, cudaFuncSetAttribute(fused_variant<PH>(v), cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
        PK_CUDA(h, cudaFuncSetAttribute(k_stage<PH, MAXT>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
        done = true;
    }
    return PK_OK;
}

template <class PH>
static int launch_fused(pk_ctx* h, Block& b, int dir, double dt, double ch, double psi_fac)
{
    if (int rc = set_smem_attr<PH>(h)) return rc;
    Geom g = make_geom(b, dir);
    Tile tl;
    int L = h->tileL[dir] > 0 ? h->tileL[dir] : DEF_L[dir];
    if (L > b.n[dir]) L = b.n[dir];
    int P = h->tileP[dir] > 0 ? h->tileP[dir] : DEF_P[dir];
    if (P > g.n1) P = g.n1;
    const int var = h->tileV[dir] >= 0 ? h->tileV[dir] : DEF_VARIANT[dir];
    const int maxt = VAR_T[var];
    int T = L + 8;
    while (P * T > maxt && P > 1) --P;
    if (P * T > maxt) return fail(h, PK_E_ARG, "fused sweep tile longer than the variant's CTA size");
    tl.P = P;
    tl.T = T;
    tl.L = L;
    tl.halo = 4;
    tl.xfast = (dir == 0);
    dim3 grid((g.n1 + P - 1) / P, (b.n[dir] + L - 1) / L, g.n2);
    size_t smem = 3ull * PH::NV * P * T * sizeof(double);
    const double dtodx1 = (0.5 * dt) / b.dl[dir];   // rk_coef(RK2_1) * dt / dl
    const double dtodx2 = (1.0 * dt) / b.dl[dir];   // rk_coef(RK2_2) * dt / dl
    std::pair<cudaEvent_t, cudaEvent_t> ev;
    if (int rc = ev_begin(h, &ev)) return fail(h, rc, "cudaEventRecord failed");
    fused_variant<PH>(var)<<<grid, P * T, smem, h->stream>>>(g, tl, b.u, b.tmp, h->pp, dtodx1, dtodx2, ch, psi_fac,
                                                            h->d_status);
    PK_CUDA(h, cudaGetLastError());
    if (int rc = ev_end(h, ev)) return fail(h, rc, "cudaEventRecord failed");
    h->launches += 1;
    h->sweep_launches += 1;
    std::swap(b.u, b.tmp);
    b.guards_stale = true;
    return PK_OK;
}

template <class PH>
static int launch_stage(pk_ctx* h, Block& b, int dir, int first, double dtodx, double ch)
{
    if (int rc = set_smem_attr<PH>(h)) return rc;
    Geom g = make_geom(b, dir);
    Tile tl;
    const int ext = b.ext[dir];
    double* uout = b.u;
    if (ext <= MAXT) {                       // whole pencil per tile: in place
        int P = MAXT / ext;
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
        if (!b.tmp) PK_CUDA(h, cudaMalloc(&b.tmp, sizeof(double) * h->nplanes * b.plane));
        uout = b.tmp;
    }
    tl.xfast = (dir == 0);
    dim3 grid((g.n1 + tl.P - 1) / tl.P, (ext + tl.L - 1) / tl.L, g.n2);
    size_t smem = 3ull * PH::NV * tl.P * tl.T * sizeof(double);
    std::pair<cudaEvent_t, cudaEvent_t> ev;
    if (int rc = ev_begin(h, &ev)) return fail(h, rc, "cudaEventRecord failed");
    k_stage<PH, MAXT><<<grid, tl.P * tl.T, smem, h->stream>>>(g, tl, b.u, uout, b.uh, h->pp, first, dtodx, ch,
                                                             h->d_status);
    PK_CUDA(h, cudaGetLastError());
    if (int rc = ev_end(h, ev)) return fail(h, rc, "cudaEventRecord failed");
    h->launches += 1;
    h->sweep_launches += 1;
    if (uout != b.u) {
        BoxGeom bg;
        for (int d = 0; d < 3; ++d) {
            bg.ext[d] = b.ext[d];
            bg.g[d] = b.g[d];
            bg.n[d] = b.n[d];
        }
        bg.plane = b.plane;
        k_copy_pencils<<<grid1d(b.plane, 256), 256, 0, h->stream>>>(bg, dir, b.tmp, b.u, h->nplanes);
        PK_CUDA(h, cudaGetLastError());
        h->launches += 1;
    }
    return PK_OK;
}

static BoxGeom box_of(const Block& b)
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

static int fill_guards_block(pk_ctx* h, Block& b)
{
    GuardArgs a;
    int f = 0, beg = 0;
    for (int d = 0; d < 3; ++d)
        for (int s = 0; s < 2; ++s) a.bnd[d][s] = b.bnd[d][s];
    for (int i = 0; i < 3; ++i)
        for (int d = 0; d < 3; ++d) a.mom_plane[i][d] = -1;
    for (f = 0; f < h->cfg.nfluids; ++f) {
        for (int d = 0; d < 3; ++d) a.mom_plane[f][d] = beg + 1 + d;
        beg += (h->cfg.fluid_kind[f] == PK_FLUID_DST) ? 4 : 5;
    }
    a.nfl = h->cfg.nfluids;
    a.nplanes = h->nplanes;
    k_fill_guards<<<grid1d(b.plane, 256), 256, 0, h->stream>>>(box_of(b), b.u, a);
    PK_CUDA(h, cudaGetLastError());
    h->launches += 1;
    b.guards_stale = false;
    return PK_OK;
}

static bool fused_ok(pk_ctx* h)
{
    if (h->cfg.integration_order != 2) return false;
    for (auto& b : h->blocks)
        for (int d = 0; d < 3; ++d)
            if (b.n[d] > 1 && (b.bnd[d][0] != PK_BND_PER || b.bnd[d][1] != PK_BND_PER)) return false;
    return true;
}

static int dispatch_fused(pk_ctx* h, Block& b, int dir, double dt, double ch, double psi_fac)
{
    if (!b.tmp) PK_CUDA(h, cudaMalloc(&b.tmp, sizeof(double) * h->nplanes * b.plane));
    if (h->phys == PHYS_MHD1) return launch_fused<PhMHD1>(h, b, dir, dt, ch, psi_fac);
    return launch_fused<PhHD1>(h, b, dir, dt, ch, psi_fac);
}

static int dispatch_stage(pk_ctx* h, Block& b, int dir, int first, double dtodx, double ch)
{
    if (!b.uh) PK_CUDA(h, cudaMalloc(&b.uh, sizeof(double) * h->nplanes * b.plane));
    if (h->phys == PHYS_MHD1) return launch_stage<PhMHD1>(h, b, dir, first, dtodx, ch);
    return launch_stage<PhHD1>(h, b, dir, first, dtodx, ch);
}

static int glm_scale(pk_ctx* h, double fac)
{
    for (auto& b : h->blocks) {
        k_scale<<<grid1d(b.plane, 256), 256, 0, h->stream>>>(b.u + (long long)(h->ib + 3) * b.plane, b.plane, fac);
        PK_CUDA(h, cudaGetLastError());
        h->launches += 1;
    }
    return PK_OK;
}

// sweep(cdim) with an optional psi damping factor folded into its last write
static int sweep_impl(pk_ctx* h, int dir, double dt, double ch, double psi_fac)
{
    if (h->blocks.empty()) return fail(h, PK_E_STATE, "no block registered");
    if (fused_ok(h)) {
        for (auto& b : h->blocks)
            if (b.n[dir] > 1)
                if (int rc = dispatch_fused(h, b, dir, dt, ch, psi_fac)) return rc;
        return PK_OK;
    }
    const int nst = h->cfg.integration_order == 1 ? 1 : 2;
    for (int s = 1; s <= nst; ++s) {
        const double rk = (h->cfg.integration_order == 1) ? 1.0 : (s == 1 ? 0.5 : 1.0);
        for (auto& b : h->blocks) {
            if (b.n[dir] <= 1) continue;
            const double dtodx = (rk * dt) / b.dl[dir];
            if (int rc = dispatch_stage(h, b, dir, s == 1, dtodx, ch)) return rc;
        }
        for (auto& b : h->blocks)
            if (int rc = fill_guards_block(h, b)) return rc;
    }
    if (h->cfg.magnetic && psi_fac != 1.0) return glm_scale(h, psi_fac);
    return PK_OK;
}

static double min_dl(pk_ctx* h, int* eff)
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
}

int pk_create(const pk_config* cfg, pk_handle* out)
{
    if (!cfg || !out) return PK_E_ARG;
    *out = nullptr;
    pk_ctx* h = new pk_ctx();
    h->cfg = *cfg;
    const pk_config& c = *cfg;
    int nvf = 0;
    bool ok = c.nfluids >= 1 && c.nfluids <= 3 && c.nb >= 2 && c.cfl > 0.0 && c.cfl <= 1.0 &&
              (c.integration_order == 1 || c.integration_order == 2);
    for (int f = 0; ok && f < c.nfluids; ++f) {
        if (c.fluid_kind[f] < 0 || c.fluid_kind[f] > 2 || (f > 0 && c.fluid_kind[f] <= c.fluid_kind[f - 1])) ok = false;
        nvf += (c.fluid_kind[f] == PK_FLUID_DST) ? 4 : 5;
        h->pp.gam[f] = (c.fluid_kind[f] == PK_FLUID_DST) ? -1.0 : c.gamma[f];
        h->pp.gam_1[f] = h->pp.gam[f] - 1.0;
    }
    ok = ok && c.limiter >= 0 && c.limiter <= 3 && c.limiter_b >= 0 && c.limiter_b <= 3;
    if (!ok) {
        delete h;
        return PK_E_ARG;
    }
    if (c.nfluids == 1 && c.fluid_kind[0] != PK_FLUID_DST && !c.magnetic) h->phys = PHYS_HD1;
    else if (c.nfluids == 1 && c.fluid_kind[0] == PK_FLUID_ION && c.magnetic) h->phys = PHYS_MHD1;
    else {
        delete h;
        return PK_E_UNSUPPORTED;
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
    std::memset(&h->ts, 0, sizeof(h->ts));
    h->ts.dt_old = -1.0;
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc(&h->d_status, sizeof(unsigned)) != cudaSuccess ||
        cudaMemset(h->d_status, 0, sizeof(unsigned)) != cudaSuccess) {
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
    for (auto& b : h->blocks) {
        cudaFree(b.u);
        cudaFree(b.uh);
        cudaFree(b.tmp);
        cudaFree(b.stage);
    }
    for (auto& p : h->ev_used) { cudaEventDestroy(p.first); cudaEventDestroy(p.second); }
    for (auto& p : h->ev_free) { cudaEventDestroy(p.first); cudaEventDestroy(p.second); }
    cudaFree(h->d_status);
    cudaFree(h->d_red);
    cudaFreeHost(h->h_red);
    cudaStreamDestroy(h->stream);
    delete h;
    return PK_OK;
}

const char* pk_last_error(pk_handle h) { return h ? h->err.c_str() : "null handle"; }

void* pk_stream(pk_handle h) { return h ? (void*)h->stream : nullptr; }

int pk_block_add(pk_handle h, const int32_t n[3], const double dl[3], const int32_t bnd[6], int32_t* id_out)
{
    if (!h || !n || !dl || !bnd) return PK_E_ARG;
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
    }
    if (h->cfg.magnetic)
        for (int d = 0; d < 3; ++d)
            if (b.n[d] > 1 && (b.bnd[d][0] != PK_BND_PER || b.bnd[d][1] != PK_BND_PER))
                return fail(h, PK_E_UNSUPPORTED, "magnetised blocks support periodic boundaries only");
    b.plane = (long long)b.ext[0] * b.ext[1] * b.ext[2];
    if (cudaMalloc(&b.u, sizeof(double) * h->nplanes * b.plane) != cudaSuccess)
        return fail(h, PK_E_NOMEM, "cudaMalloc of the block state failed");
    PK_CUDA(h, cudaMemsetAsync(b.u, 0, sizeof(double) * h->nplanes * b.plane, h->stream));
    h->blocks.push_back(b);
    if (id_out) *id_out = (int32_t)h->blocks.size() - 1;
    const int need = (int)h->blocks.size() * 12;
    if (need > h->red_cap) {
        cudaFree(h->d_red);
        cudaFreeHost(h->h_red);
        h->red_cap = need + 120;
        PK_CUDA(h, cudaMalloc(&h->d_red, sizeof(unsigned long long) * h->red_cap));
        PK_CUDA(h, cudaMallocHost(&h->h_red, sizeof(unsigned long long) * h->red_cap));
    }
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
    if (layout == PK_LAYOUT_SOA) {
        PK_CUDA(h, cudaMemcpyAsync(b->u, u, sizeof(double) * h->nvf * nc, cudaMemcpyHostToDevice, h->stream));
        if (h->cfg.magnetic) {
            PK_CUDA(h, cudaMemcpyAsync(b->u + (long long)h->ib * nc, bf, sizeof(double) * 3 * nc, cudaMemcpyHostToDevice, h->stream));
            PK_CUDA(h, cudaMemcpyAsync(b->u + (long long)(h->ib + 3) * nc, psi, sizeof(double) * nc, cudaMemcpyHostToDevice, h->stream));
        }
    } else if (layout == PK_LAYOUT_FORTRAN) {
        if (!b->stage) PK_CUDA(h, cudaMalloc(&b->stage, sizeof(double) * h->nvf * nc));
        PK_CUDA(h, cudaMemcpyAsync(b->stage, u, sizeof(double) * h->nvf * nc, cudaMemcpyHostToDevice, h->stream));
        k_aos_to_soa<<<grid1d(nc, 256), 256, 0, h->stream>>>(b->stage, b->u, nc, h->nvf, 0, nc);
        PK_CUDA(h, cudaGetLastError()); h->launches += 1;
        if (h->cfg.magnetic) {
            // the staging buffer is reused once the first conversion has run (same stream)
            PK_CUDA(h, cudaMemcpyAsync(b->stage, bf, sizeof(double) * 3 * nc, cudaMemcpyHostToDevice, h->stream));
            k_aos_to_soa<<<grid1d(nc, 256), 256, 0, h->stream>>>(b->stage, b->u, nc, 3, h->ib, nc);
            PK_CUDA(h, cudaGetLastError()); h->launches += 1;
            PK_CUDA(h, cudaMemcpyAsync(b->u + (long long)(h->ib + 3) * nc, psi, sizeof(double) * nc, cudaMemcpyHostToDevice, h->stream));
        }
    } else {
        return fail(h, PK_E_ARG, "unknown layout");
    }
    return PK_OK;
}

int pk_download(pk_handle h, int32_t id, double* u, double* bf, double* psi, int32_t layout)
{
    Block* b;
    if (int rc = get_block(h, id, &b)) return rc;
    if (!u || (h->cfg.magnetic && (!bf || !psi))) return fail(h, PK_E_ARG, "null array");
    if (b->guards_stale)
        if (int rc = fill_guards_block(h, *b)) return rc;
    const long long nc = b->plane;
    if (layout == PK_LAYOUT_SOA) {
        PK_CUDA(h, cudaMemcpyAsync(u, b->u, sizeof(double) * h->nvf * nc, cudaMemcpyDeviceToHost, h->stream));
        if (h->cfg.magnetic) {
            PK_CUDA(h, cudaMemcpyAsync(bf, b->u + (long long)h->ib * nc, sizeof(double) * 3 * nc, cudaMemcpyDeviceToHost, h->stream));
            PK_CUDA(h, cudaMemcpyAsync(psi, b->u + (long long)(h->ib + 3) * nc, sizeof(double) * nc, cudaMemcpyDeviceToHost, h->stream));
        }
    } else if (layout == PK_LAYOUT_FORTRAN) {
        if (!b->stage) PK_CUDA(h, cudaMalloc(&b->stage, sizeof(double) * h->nvf * nc));
        k_soa_to_aos<<<grid1d(nc, 256), 256, 0, h->stream>>>(b->u, b->stage, nc, h->nvf, 0, nc);
        PK_CUDA(h, cudaGetLastError()); h->launches += 1;
        PK_CUDA(h, cudaMemcpyAsync(u, b->stage, sizeof(double) * h->nvf * nc, cudaMemcpyDeviceToHost, h->stream));
        if (h->cfg.magnetic) {
            PK_CUDA(h, cudaStreamSynchronize(h->stream));   // the staging buffer is reused for b
            k_soa_to_aos<<<grid1d(nc, 256), 256, 0, h->stream>>>(b->u, b->stage, nc, 3, h->ib, nc);
            PK_CUDA(h, cudaGetLastError()); h->launches += 1;
            PK_CUDA(h, cudaMemcpyAsync(bf, b->stage, sizeof(double) * 3 * nc, cudaMemcpyDeviceToHost, h->stream));
            PK_CUDA(h, cudaMemcpyAsync(psi, b->u + (long long)(h->ib + 3) * nc, sizeof(double) * nc, cudaMemcpyDeviceToHost, h->stream));
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
    const double dtodx = (rk * dt) / b->dl[dir];   // rk_coef(istep) * dt / cg%dl(ddim)
    return dispatch_stage(h, *b, dir, first, dtodx, chspeed);
}

int pk_fill_guards(pk_handle h)
{
    if (!h) return PK_E_ARG;
    for (auto& b : h->blocks)
        if (int rc = fill_guards_block(h, b)) return rc;
    return PK_OK;
}

int pk_sweep(pk_handle h, int32_t cdim, double dt, double chspeed)
{
    if (!h) return PK_E_ARG;
    if (cdim < 1 || cdim > 3) return fail(h, PK_E_ARG, "cdim must be 1..3");
    return sweep_impl(h, cdim - 1, dt, chspeed, 1.0);
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
    for (int i = 0; i < nb; ++i) {
        Block& b = h->blocks[i];
        const long long ncell = (long long)b.n[0] * b.n[1] * b.n[2];
        k_cfl<<<grid1d(ncell, 256), 256, 0, h->stream>>>(box_of(b), b.u, a, h->d_red + 12 * i);
        PK_CUDA(h, cudaGetLastError());
        h->launches += 1;
    }
    PK_CUDA(h, cudaMemcpyAsync(h->h_red, h->d_red, sizeof(unsigned long long) * 12 * nb, cudaMemcpyDeviceToHost, h->stream));
    PK_CUDA(h, cudaStreamSynchronize(h->stream));
    double dt = DBL_MAX, c_all = 0.0;                  // timestep.F90:161-162
    for (int i = 0; i < nb; ++i) {
        const Block& b = h->blocks[i];
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

int pk_time_step(pk_handle h, double* dt_out)
{
    if (!h) return PK_E_ARG;
    double dt, c_all;
    h->ts.dt_old = h->ts.dt;                          // timestep.F90:158
    if (int rc = pk_timestep_raw(h, &dt, &c_all)) return rc;
    const pk_config& c = h->cfg;
    if (h->ts.nstep < 1) {                            // :200-208
        if (c.dt_initial > 0.0) dt = (c.dt_initial < dt) ? c.dt_initial : dt;
        else if (c.dt_initial < 0.0) {
            const double x = -c.dt_initial * dt;
            dt = (x < dt) ? x : dt;
        }
    } else if (h->ts.dt_old > 0.0) {
        const double x = h->ts.dt_old * c.dt_max_grow;
        dt = (x < dt) ? x : dt;
    }
    h->ts.c_all = c_all;
    if (dt < c.dt_min) {                              // :213-219
        h->ts.dt = dt;
        if (dt_out) *dt_out = dt;
        return fail(h, PK_E_DTMIN, "dt < dt_min");
    }
    const double rem = c.tend - h->ts.t;              // :224
    const double cap = (0.5 * rem) + ((2.0 * DBL_EPSILON) * rem);
    dt = (c.dt_max < dt) ? c.dt_max : dt;
    dt = (cap < dt) ? cap : dt;
    h->ts.dt = dt;
    if (dt_out) *dt_out = dt;
    return PK_OK;
}

int pk_fluid_update(pk_handle h)
{
    if (!h) return PK_E_ARG;
    const double dt = h->ts.dt;
    int eff;
    const double mdl = min_dl(h, &eff);
    if (h->cfg.magnetic) {                            // update_chspeed, hdc.F90:112-119
        double ch = DBL_MAX;
        if (eff) {
            const double x = (h->cfg.cfl_glm * mdl) / dt;
            ch = (x < ch) ? x : ch;
        }
        h->ts.chspeed = ch;
    }
    double fac = 1.0;
    if (h->cfg.magnetic) {                            // glmdamping, hdc.F90:310-330
        double f = 0.0;
        if (eff) {
            const double x = (h->cfg.glm_alpha * h->ts.chspeed) / (mdl / dt);
            f = (x > f) ? x : f;
        }
        fac = std::exp(-f);
    }
    int dirs[3], nd = 0;
    for (int d = 0; d < 3; ++d) {
        bool has = false;
        for (auto& b : h->blocks) has = has || b.n[d] > 1;
        if (has && !h->cfg.skip_sweep[d]) dirs[nd++] = d;
    }
    for (int half = 0; half < 2; ++half) {            // fluidupdate.F90:115-130
        h->ts.t = h->ts.t + dt;
        for (int s = 0; s < nd; ++s) {
            const int d = half == 0 ? dirs[s] : dirs[nd - 1 - s];
            const double pf = (h->cfg.magnetic && s == nd - 1) ? fac : 1.0;
            if (int rc = sweep_impl(h, d, dt, h->ts.chspeed, pf)) return rc;
        }
        if (h->cfg.magnetic && nd == 0)
            if (int rc = glm_scale(h, fac)) return rc;
    }
    return PK_OK;
}

int pk_run(pk_handle h, int32_t nsteps)
{
    if (!h) return PK_E_ARG;
    for (int s = 0; s < nsteps; ++s) {
        if (!(h->ts.t < h->cfg.tend)) break;
        if (int rc = pk_time_step(h, nullptr)) return rc;
        if (int rc = pk_fluid_update(h)) return rc;
        h->ts.nstep += 1;
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

int pk_set_tile(pk_handle h, int32_t dir, int32_t pencils, int32_t length, int32_t variant)
{
    if (!h || dir < 0 || dir > 2 || pencils < 0 || length < 0 || variant < -1 || variant >= NVARIANT) return PK_E_ARG;
    const int maxt = VAR_T[variant >= 0 ? variant : DEF_VARIANT[dir]];
    if (length > 0 && length + 8 > maxt) return fail(h, PK_E_ARG, "length + 8 exceeds the variant's CTA size");
    h->tileP[dir] = pencils;
    h->tileL[dir] = length;
    h->tileV[dir] = variant;
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
