// pk_internal.h -- host-side state of a library handle, shared by the C ABI
// (pk_api.cu) and the per-physics launch units (pk_phys_*.cu).
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <utility>
#include <vector>

#include "../../include/piernik_b200.h"
#include "pk_aux.cuh"
#include "pk_kernels.cuh"
#include "pk_levels.h"

namespace pk {

// Launch-bound variants of the fused sweep (threads per CTA, CTAs per SM):
// the register budget the compiler may use is 65536 / (threads * CTAs);
// tighter budgets trade spills for resident warps.  The autotuner picks one
// per direction.
// Variant VAR_STAGED is the TMA-staged whole-pencil kernel (pk_staged.cuh:
// two pencils per 256-thread CTA, two CTAs per SM).
constexpr int NVARIANT = 8;
constexpr int VAR_T[NVARIANT] = {320, 256, 256, 128, 128, 192, 512, 256};
constexpr int VAR_B[NVARIANT] = {1, 1, 2, 3, 4, 2, 1, 2};
constexpr int VAR_STAGED = 7;
constexpr int STAGE_MAXT = 320;       // threads per CTA of the stage kernel
constexpr int UNSPLIT_MAXT = 256;     // threads per CTA of the unsplit flux kernel (two CTAs per SM)
// launch-bound variants of the batched stage kernel (threads per CTA, CTAs per SM)
constexpr int NSTAGE_VARIANT = 4;
constexpr int SV_T[NSTAGE_VARIANT] = {320, 128, 192, 384};
constexpr int SV_B[NSTAGE_VARIANT] = {1, 3, 2, 1};
constexpr int W3_VARIANT = 2;          // interpol_str = 'weno3' runs this launch-bound variant only

struct Block {
    int n[3], g[3], ext[3];
    double dl[3];
    int bnd[3][2];
    long long plane = 0;
    double* buf[2] = {nullptr, nullptr};   // state and its ping-pong partner
    double* uh = nullptr;                  // stage path: state at the start of the step (cg%w(uh))
    double* stage = nullptr;               // host-layout conversion buffer
    bool guards_stale = false;             // fused sweeps read periodic images and never store guards
    double* retry = nullptr;               // copy of the state at the start of a step (cflcontrol = redo)
    int seg_len = 0;                       // independent instances stacked along z: cells per instance
    long long off[3] = {0, 0, 0};          // first interior cell on the level's cell grid (connected domains)
    bool placed = false;
    int level = 0;                         // refinement level (0: base)
    FcArgs fc[3] = {};                     // fine/coarse flux couplings per sweep direction (device)
    unsigned char* leaf = nullptr;         // device interior leaf mask (null: every cell is a leaf)
    long long leaf_cells = -1;             // cells of the mask set (-1: all)
    double* flux[3] = {nullptr, nullptr, nullptr};   // unsplit scheme: face fluxes per direction
    unsigned char* flag = nullptr;         // refinement flag map (ext cells), pk_mark_refinement
};

// the per-block stage kernel sweeps whole pencils in place where they fit
// the CTA (for y and z sweeps only when four or more neighbouring pencils
// share it, so that the loads stay coalesced), else chunks with a 2-cell halo
// out of place into the ping-pong buffer
inline bool stage_chunked(const Block& b, int dir)
{
    const int ext = b.ext[dir], n1 = b.n[dir == 0 ? 1 : 0];
    return !(ext <= STAGE_MAXT && (dir == 0 || STAGE_MAXT / ext >= 4 || n1 < 4));
}

struct pk_dir_tile { int P, L, V; };

// scalars of one recorded step of the differentiable path
struct StepRec {
    double dt, ch, fac;
};

// device copy of a segment list with its cell count
struct XSegList {
    XSegDev* dev = nullptr;
    int n = 0;
    long long total = 0;
};

// the halo traffic with one other rank
struct XPeerDev {
    int rank = -1;
    XSegList send, recv;
    XSegList send_dir[3], recv_dir[3];   // the face boxes along one direction (seg_face_dir)
};

// a block held by another rank (connected domains spanning ranks)
struct RemoteBlock {
    int owner;
    int n[3];
    long long off[3];
};

// work list of the batched sweep for one direction
struct BatchList {
    std::vector<WorkItem> host;
    WorkItem* dev = nullptr;
    int n = 0;
};

// work list of the batched stage for one direction and level
struct StageList {
    StageItem* dev = nullptr;
    int n = 0;
    size_t smem = 0;
};

}  // namespace pk

struct pk_ctx {
    pk_config cfg;
    pk::PhysParams pp;
    int phys = 0;
    int nvf = 0, nplanes = 0, ib = 0;
    std::vector<pk::Block> blocks;
    int cur = 0;                        // which of Block::buf holds the state (all blocks alike)
    cudaStream_t stream = nullptr;
    unsigned* d_status = nullptr;
    unsigned* d_counter = nullptr;      // work-list counters of the batched sweep (one per launch slot)
    unsigned long long* d_red = nullptr;
    unsigned long long* d_ch = nullptr;     // the gas-based chspeed maximum (ch_grid = 0)
    unsigned long long* h_red = nullptr;
    int red_cap = 0;
    pk::StepParams* d_step = nullptr;   // device copy of the step scalars (one per instance)
    pk::StepParams* h_step = nullptr;   // pinned host copy
    int ninst = 1;                      // independent instances stacked along z in the one block
    std::vector<pk_time_state> its;     // their time states (ninst > 1)
    pk::BlockDesc* d_inst[2] = {nullptr, nullptr};   // the instances as CFL blocks, per parity
    pk::BlockDesc* d_desc[2] = {nullptr, nullptr};   // block tables for cur = 0 / 1
    bool batch_dirty = true;
    pk::BatchList batch[3];
    std::vector<pk::StageList> sbatch[3];       // batched stage per direction, per level
    bool stage_batched = false;                 // every block's pencils fit one stage CTA
    // refined domains: every level's stage items and the restriction chunks
    // between them as one work list per direction (k_stage_refined)
    pk::RefItem* rdev[3] = {nullptr, nullptr, nullptr};
    int rn[3] = {0, 0, 0};
    size_t rsmem[3] = {0, 0, 0};
    unsigned* d_rcount = nullptr;               // its counters (1 + 2 levels), zeroed before each launch
    int rcount_n = 0;
    bool refined_one_launch = false;            // pk_set_refined_launch
    double* d_eglm = nullptr;                   // E-GLM scratch: divB and grad(psi), 4 planes of the largest block
    long long eglm_plane = 0;
    int stage_variant = 0;                      // launch-bound variant of k_stage_batched (SV_T / SV_B)
    pk::FcArgs* d_fcargs[3] = {nullptr, nullptr, nullptr};   // per block flux couplings (refined domains)
    pk_time_state ts;
    std::string err;
    int tileP[3] = {0, 0, 0}, tileL[3] = {0, 0, 0}, tileV[3] = {-1, -1, -1};
    int arith = 0;                      // PK_ARITH_*: the fused / batched sweeps' arithmetic
    int batched = 0;                    // 1: sweep all blocks in one persistent launch
    int batch_variant = 2;              // launch-bound variant of the batched kernel
    int batch_L = 56;                   // longest chunk of the batched tiles
    int batch_circ = 1;                 // sweep pencils that fit the CTA whole (no halo)
    long long launches = 0;             // kernels of this library launched on the handle's stream
    bool profiling = false;             // bracket sweep kernels with CUDA events
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev_used, ev_free;
    cudaGraph_t graph = nullptr;        // captured sweeps of one step (pk_run with graphs)
    cudaGraphExec_t graph_exec = nullptr;
    int use_graph = 0;
    long long graph_kernels = 0;        // kernel nodes of the captured step
    // same-level domain of connected blocks (pk_set_domain / pk_block_place)
    bool connected = false;
    long long dom[3] = {1, 1, 1};
    int dom_periodic[3] = {0, 0, 0};
    bool x_dirty = true;                // the exchange plan must be rebuilt
    bool x_ptrs_dirty = true;           // block buffers changed: rebuild the pointer tables
    pk::XSegList xlocal;                // copies between this rank's blocks
    pk::XSegList xlocal_dir[3];         // the same restricted to face boxes along one direction
    bool x_dir = false;                 // the per-direction lists are built (single-level domains)
    std::vector<pk::XPeerDev> xpeers;   // copies to and from each other rank
    std::vector<pk::RemoteBlock> remote;
    pk::XPtr* d_xptr[2] = {nullptr, nullptr};   // block states of parity 0 / 1
    // refined domains (pk_block_place_level): the fine/coarse couplings on the device
    int max_level = 0;
    pk::PRunDev* d_runs = nullptr;              // prolongation rows, by fine level
    long long* d_run_start = nullptr;           // running cell count of each row within its level
    std::vector<long long> run_beg;             // rows of fine level L: [run_beg[L], run_beg[L+1])
    std::vector<long long> run_cells;           // guard cells prolonged into level L
    int* d_fc_int[3] = {nullptr, nullptr, nullptr};          // per-pencil slot tables, in faces, flux sources
    double* d_in_flux[3] = {nullptr, nullptr, nullptr};      // restricted fluxes per in slot
    double* d_out_flux[3] = {nullptr, nullptr, nullptr};     // fine boundary fluxes per out slot
    const int* d_src[3] = {nullptr, nullptr, nullptr};
    std::vector<int> in_level_beg[3];           // in slots of coarse level L: [in_level_beg[L], in_level_beg[L+1])
    double fc_scale = 1.0;                      // 1 / 2**(eff_dim - 1)
    pk::ProlongCoef pro_u{}, pro_b{};           // prolongation stencils of the fluids and of B / psi
    pk::RBoxDev* d_rbox = nullptr;              // restriction targets, by fine level
    long long* d_rbox_start = nullptr;          // running cell count of each box within its level
    std::vector<int> rbox_beg;                  // boxes of fine level L: [rbox_beg[L], rbox_beg[L+1])
    std::vector<long long> rbox_cells;          // coarse cells restricted from level L
    int eff_dim = 3;
    // guard refresh before a stage of the interior-trimmed stage kernel along
    // direction d: only the cells it reads (build_partial_refresh)
    struct Partial {
        pk::XSegList segs;
        pk::PRunDev* runs = nullptr;
        long long* run_start = nullptr;
        std::vector<long long> run_beg, run_cells;
        bool ok = false;
    } part[3];
    pk_halo_fn halo_cb = nullptr;       // moves the halo of other ranks (host callback)
    pk_reduce_fn reduce_cb = nullptr;   // min / max over ranks for the time step
    void* comm_ctx = nullptr;
    // differentiable path (single block, fused sweeps)
    int adjL[3] = {0, 0, 0};            // owned cells per pencil of the adjoint tiles, per direction (0: default)
    int adjV[3] = {-1, -1, -1};         // launch-bound variant of the adjoint kernels per direction (-1: default)
    std::vector<pk::StepRec> grad_steps;        // dt, chspeed, damping of each recorded step
    std::vector<double*> grad_ckpt;             // checkpointed states (every grad_every steps)
    int grad_every = 0;
    double* lam = nullptr;                      // adjoint of the state (structure of arrays)
    double* lam_tmp = nullptr;
    std::vector<double*> grad_pool;             // outputs of a recomputed segment's sweeps
    std::vector<double*> grad_star;             // their stage-1 states
    std::vector<unsigned short*> grad_flags;    // their floor records
    double* lam_m1 = nullptr;                   // scratch state of the adjoint sweep
    pk_time_state grad_ts0;                     // time state at the start of the recording
};

namespace pk {

// multiprocessors of the current device (looked up once per device); 1-D
// grid-stride kernels launch at most 16 CTAs of 256 threads per SM
inline int sm_count()
{
    static int cache[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
    if (!cache[dev]) {
        int n = 0;
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n < 1) n = 148;
        cache[dev] = n;
    }
    return cache[dev];
}

inline long long grid_cap() { return (long long)sm_count() * 16; }

int fail(pk_ctx* h, int code, const std::string& msg);
int ev_begin(pk_ctx* h, std::pair<cudaEvent_t, cudaEvent_t>* p);
int ev_end(pk_ctx* h, const std::pair<cudaEvent_t, cudaEvent_t>& p);
Geom make_geom(const Block& b, int dir);

// launches of one physics configuration (pk_phys_*.cu)
struct PhysOps {
    int nv;
    int (*prepare)(pk_ctx* h);      // kernel attributes; called before any launch or graph capture
    int (*fused)(pk_ctx* h, Block& b, int dir, int apply_fac);
    int (*stage)(pk_ctx* h, Block& b, int dir, int first, double rk);           // dt, ch from d_step
    int (*stage_batched)(pk_ctx* h, int dir, int level, int first, double rk);  // all blocks of a level
    int (*stage_refined)(pk_ctx* h, int dir, int first, double rk);             // all levels, one launch
    int (*batched)(pk_ctx* h, int dir, int apply_fac, unsigned* counter);
    int (*fused_ptr)(pk_ctx* h, Block& b, int dir, int apply_fac, const double* in, double* out);
    int (*fused_rec)(pk_ctx* h, Block& b, int dir, int apply_fac, const double* in, double* out, double* ustar,
                     unsigned short* flags);
    int (*adj)(pk_ctx* h, Block& b, int dir, int apply_fac, const double* uin, const double* ustar,
               const double* uout, const unsigned short* flags, const double* lam_out, double* lam_in, double* m1);
    int (*unsplit_flux)(pk_ctx* h, Block& b, int dir, const double* in, double* F);
    int (*unsplit_apply)(pk_ctx* h, Block& b, const double* S, double* T, double rk, int last);
};

// the fused and batched sweeps in the tolerance-mode arithmetic (pk_fast_*.cu,
// compiled with multiply-add contraction; pk_set_arithmetic)
struct FastOps {
    int (*prepare)(pk_ctx* h);
    int (*fused)(pk_ctx* h, Block& b, int dir, int apply_fac);
    int (*batched)(pk_ctx* h, int dir, int apply_fac, unsigned* counter);
};

const FastOps* fast_ops_hd1();
const FastOps* fast_ops_hd2();
const FastOps* fast_ops_mhd1();
const FastOps* fast_ops_mhd2();
const FastOps* fast_ops_mhd3();

const PhysOps* ops_hd1();
const PhysOps* ops_hd2();
const PhysOps* ops_mhd1();
const PhysOps* ops_mhd2();
const PhysOps* ops_mhd3();

}  // namespace pk

#define PK_CUDA(h, call)                                                                      \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess) {                                                              \
            (h)->err = std::string(#call) + ": " + cudaGetErrorString(e_);                   \
            return PK_E_CUDA;                                                                 \
        }                                                                                     \
    } while (0)
