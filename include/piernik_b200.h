/*
 * piernik_b200.h -- C ABI of the B200 split-sweep library (libpiernik_b200.so).
 *
 * The library replaces PIERNIK's RIEMANN_SPLIT fluid-update hot path: the
 * per-block Riemann solve (solve_cg_riemann), the directional sweep with its
 * RK2 stages and guardcell refresh (sweep, update_boundaries), the CFL time
 * step reduction (time_step / timestep_fluid), the GLM psi speed and damping
 * (update_chspeed, glmdamping) and the XYZ/ZYX pair of time steps
 * (fluid_update_full).  All arithmetic is IEEE binary64.
 *
 * Conventions: every entry point returns PK_OK (0) or a negative PK_E* code;
 * pk_last_error() gives a one-line message.  No entry point aborts the
 * process and no kernel traps: numerical trouble (negative density or
 * internal energy) is reported through pk_status().  One CUDA stream per
 * handle; a handle must not be used from two host threads at once.
 *
 * Array layouts accepted by pk_upload/pk_download:
 *   PK_LAYOUT_FORTRAN  the reference's named arrays with guard cells:
 *                      u(nvar, i, j, k), b(3, i, j, k), psi(i, j, k),
 *                      column-major, i over lhn(x), j over lhn(y), k over lhn(z)
 *                      (src/grid/grid_container_base.F90 lhn extents)
 *   PK_LAYOUT_SOA      u[v][k][j][i], b[d][k][j][i], psi[k][j][i], same extents
 * Component order of u is the reference's flind order: for each fluid
 * (ionized, neutral, dust) [dn, mx, my, mz, (en)] (fluids/fluidtypes.F90:279-330).
 */
#ifndef PIERNIK_B200_H
#define PIERNIK_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PK_ABI_VERSION 6

enum {
    PK_OK = 0,
    PK_E_ARG = -1,         /* invalid argument / configuration */
    PK_E_CUDA = -2,        /* CUDA runtime error (message in pk_last_error) */
    PK_E_NOMEM = -3,       /* device allocation failed */
    PK_E_UNSUPPORTED = -4, /* configuration not provided by this build */
    PK_E_STATE = -5,       /* call out of order (e.g. no block registered) */
    PK_E_DTMIN = -6        /* dt < dt_min: the reference calls write_crashed */
};

enum { PK_FLUID_ION = 0, PK_FLUID_NEU = 1, PK_FLUID_DST = 2 };
enum { PK_LIM_VANLEER = 0, PK_LIM_MINMOD = 1, PK_LIM_MONCEN = 2, PK_LIM_SUPERBEE = 3 };
enum { PK_BND_PER = 0, PK_BND_OUT = 1, PK_BND_REF = 2 };
enum { PK_LAYOUT_FORTRAN = 0, PK_LAYOUT_SOA = 1 };
enum { PK_ST_DN_NEGATIVE = 1, PK_ST_EI_NEGATIVE = 2,
       PK_ST_TIMEOUT = 4 /* a kernel's bounded wait on an asynchronous copy gave up (its tile was not swept) */ };
/* RK stage identifiers, numerically equal to the reference's istep enumerators
 * (src/base/constants.F90:230-238) */
enum { PK_EULER = 10000, PK_RK2_1 = 10001, PK_RK2_2 = 10002 };

/* NUMERICAL_SETUP / FLUID_* / END_CONTROL parameters the path reads
 * (src/base/global.F90:118-120 and defaults :196-260). */
typedef struct pk_config {
    int32_t nfluids;            /* 1..3, in flind order */
    int32_t fluid_kind[3];      /* PK_FLUID_* */
    double gamma[3];            /* FLUID_*: gamma (dust: ignored, -1 used) */
    int32_t magnetic;           /* MAGNETIC with divB_0 = 'HDC' (B + psi) */
    int32_t limiter;            /* NUMERICAL_SETUP: limiter   (PK_LIM_*) */
    int32_t limiter_b;          /* NUMERICAL_SETUP: limiter_b (PK_LIM_*) */
    int32_t use_smalld, use_smallei, disallow_negatives;
    double smalld, smallei;
    double cfl, cfl_glm, glm_alpha;
    int32_t integration_order;  /* 1 or 2 */
    int32_t nb;                 /* guard cells (dom%nb) */
    double dt_initial, dt_max_grow, dt_min, dt_max;
    double tend;                /* END_CONTROL: tend */
    int32_t skip_sweep[3];
    /* step retry: cflcontrol (PK_CFL_*), cfl_max (sanitised as global.F90:304),
     * dt_shrink, max_redostep_attempts (global.F90:218,233,245,258) */
    int32_t cflcontrol;
    double cfl_max, dt_shrink;
    int32_t max_redostep_attempts;
    /* interpol_str (global.F90:220): PK_INTERP_LINEAR or PK_INTERP_WENO3, and
     * w_epsilon (:255) for WENO3 */
    int32_t interpolation;
    double w_epsilon;
    /* solver_str (global.F90:423-437): PK_SOLVER_SPLIT (RIEMANN_SPLIT) or
     * PK_SOLVER_UNSPLIT (RIEMANN_UNSPLIT, src/scheme/unsplit_schemes) */
    int32_t solver;
    /* ord_fluid_prolong, ord_mag_prolong (global.F90:113-114, defaults O_INJ
     * and O_I2 :259-260): the reference's prolongation orders of refined
     * domains' guard cells, PK_O_* (0 injection, 1 linear, 2..6 integral,
     * -2..-6 direct); fluids accept injection or linear only (others degrade
     * to injection, global.F90:561-566); 2 x the stencil range (0 for
     * injection, 1 for orders +-1..2, 2 for 3..4, 3 for 5..6) must not exceed nb */
    int32_t ord_fluid_prolong, ord_mag_prolong;
    /* ch_grid (global.F90:111, default .true. :254): 1 = chspeed from the
     * grid, cfl_glm * min(dl) / dt; 0 = from the gas, the maximum over leaf
     * cells of point_chspeed (hdc.F90:118-131,197-268), reduced over ranks
     * with MAX (one device reduction per step) */
    int32_t ch_grid;
    /* use_eglm (global.F90:109, default .false. :252): the E-GLM sources of
     * hdc.F90:355-457 after each triple of sweeps, before the psi damping --
     * on the ionized fluid, m -= dt divB B, B -= dt divB v, E -= dt (divB v.B
     * - B.grad psi), psi -= dt v.grad psi, with divB and grad psi of order 2
     * from the cells' neighbours (the guard cells refreshed around them).
     * RIEMANN_SPLIT only (the reference stops otherwise, hdc.F90:388), and
     * here on single-level domains without stacked instances, outside the
     * differentiable path (ABI version 6) */
    int32_t use_eglm;
} pk_config;

#define PK_SOLVER_SPLIT   0
#define PK_SOLVER_UNSPLIT 1

#define PK_INTERP_LINEAR 0
#define PK_INTERP_WENO3  1

#define PK_CFL_NONE 0           /* no check */
#define PK_CFL_WARN 1           /* stepcfl computed each step (timestep.F90:317-360), no retry */
#define PK_CFL_REDO 2           /* a step whose effective CFL exceeds cfl_max, or that made
                                   unwanted negatives, is redone with dt x dt_shrink^attempt
                                   (timestep_retry.F90:repeat_fluidstep) -- the reference default */
#define PK_CFL_FLEX 3           /* 'flex': redone as REDO, with dt x cfl_max / stepcfl (x dt_shrink
                                   from the second attempt on) (timestep.F90:81-84,347-351) */
#define PK_CFL_AUTO 4           /* 'auto': cfl_auto in the main time step, dt x cfl_c with
                                   cfl_c = min(1, (cfl_c + min(1, stepcfl_old / stepcfl * dt /
                                   dt_old)) / 2) (timestep.F90:85-86,368-405), no retry */

/* Time-integration state the reference keeps in module global (global.F90). */
typedef struct pk_time_state {
    double t, dt, dt_old, c_all, chspeed;
    int32_t nstep;
    /* step retry state (global.F90: dt_full, dt_cur_shrink, t_saved, nstep_saved,
     * tstep_attempt; timestep_pub: c_all_old, stepcfl; repeatstep: repeat_step) */
    double dt_full, c_all_old, dt_cur_shrink, stepcfl, t_saved;
    int32_t nstep_saved, tstep_attempt, repeat_step, redone;
    /* cfl_c of cfl_auto (timestep_pub, initially one; a 0 here is read as one) */
    double cfl_c;
} pk_time_state;

typedef struct pk_ctx* pk_handle;

/* Fill cfg with the reference defaults (global.F90:196-260, ionized gamma 5/3). */
void pk_config_default(pk_config* cfg);

/* Create / destroy a library instance on the current CUDA device. */
int pk_create(const pk_config* cfg, pk_handle* out);
int pk_destroy(pk_handle h);
const char* pk_last_error(pk_handle h);
int pk_abi_version(void);

/* Register a block (grid_container): n interior cells, cell sizes dl, external
 * boundary types per direction and side.  Single-block runs with periodic
 * boundaries are swept by the fused two-stage kernel. */
int pk_block_add(pk_handle h, const int32_t n[3], const double dl[3], const int32_t bnd[6], int32_t* id_out);

/* Free block id; the ids above it move down by one.  With pk_block_add,
 * pk_block_place_level, pk_restrict and pk_prolong_block a host regrids a
 * refined domain (the cg removal of refinement_update.F90 derefinement).
 * Refused while the differentiable path holds checkpoints. */
int pk_block_remove(pk_handle h, int32_t id);

/* Copy a block's u (all fluids), b and psi between host and device.
 * b/psi are ignored when the run is not magnetised.  Guard cells come back as
 * the last stage left them; after fused sweeps (which read periodic images and
 * never store guards) they are refreshed before the copy. */
int pk_upload(pk_handle h, int32_t id, const double* u, const double* b, const double* psi, int32_t layout);
int pk_download(pk_handle h, int32_t id, double* u, double* b, double* psi, int32_t layout);

/* solve_cg(cg, ddim, istep) for one block and one RK stage on the device
 * copy: replaces the procedure pointer target solve_cg_riemann
 * (src/scheme/sweeps.F90:138-153,245; Riemann_Solver/solve_cg_riemann.F90:68-107).
 * ddim is 1..3 (xdim..zdim), istep is PK_EULER / PK_RK2_1 / PK_RK2_2.
 * Guard cells are not refreshed (the caller's update_boundaries does that,
 * or pk_fill_guards). */
int pk_solve_cg(pk_handle h, int32_t id, int32_t ddim, int32_t istep, double dt, double chspeed);

/* update_boundaries for all blocks (sweeps.F90:66-107, single level). */
int pk_fill_guards(pk_handle h);

/* sweep(cdim): all RK stages over all blocks with guardcell refresh
 * (src/scheme/sweeps.F90:114-279); cdim is 1..3. */
int pk_sweep(pk_handle h, int32_t cdim, double dt, double chspeed);

/* glmdamping: psi *= fac on every block (Riemann_Solver/hdc.F90:289-349). */
int pk_glm_damp(pk_handle h, double fac);

/* timestep_fluid over all fluids and blocks, before clamps
 * (src/base/timestep.F90:431-495): dt = cfl*min_d(dl_d/max c_d), c_all. */
int pk_timestep_raw(pk_handle h, double* dt_out, double* c_all_out);

/* time_step(dt, flind, .true.) with the sanity clamps (timestep.F90:112-240);
 * updates the handle's pk_time_state.  Returns PK_E_DTMIN when dt < dt_min. */
int pk_time_step(pk_handle h, double* dt_out);

/* fluid_update_full (src/scheme/fluidupdate.F90:99-136): update_chspeed,
 * X->Y->Z sweeps, glmdamping, Z->Y->X sweeps, glmdamping; t += 2 dt.
 * With PK_SOLVER_UNSPLIT: fluid_update_unsplit (unsplit_fluidupdate.F90:
 * 45-126): update_chspeed, glmdamping over dt/2, t += dt, one unsplit sweep
 * (every stage: the face fluxes of all directions from the same state, the
 * x, y, z flux differences applied in turn, sources and floors;
 * unsplit_sweeps.F90:104-189), glmdamping over dt/2.  The unsplit scheme
 * runs on single, independent, connected and refined blocks of one rank
 * (refined: the fine/coarse flux replacement of fc_fluxes_unsplit.F90 and
 * the guard update of each stage's array, levels as the split scheme). */
int pk_fluid_update(pk_handle h);

/* nsteps iterations of the reference main loop body (time_step +
 * fluid_update, piernik.F90:125-213 without I/O); stops at t >= tend. */
int pk_run(pk_handle h, int32_t nsteps);

int pk_get_time_state(pk_handle h, pk_time_state* st);
int pk_set_time_state(pk_handle h, const pk_time_state* st);

/* OR of PK_ST_* bits raised since the last call; clears them. */
int pk_status(pk_handle h, uint32_t* flags);

/* Wait for all work of the handle's stream. */
int pk_sync(pk_handle h);

/* Tile shape of the fused sweep for direction d (0..2): P pencils per CTA,
 * L output cells per pencil (the CTA also computes a 4-cell halo each side),
 * and the launch-bound variant (register budget) of the kernel, -1 for the
 * default.  Used by the autotuner; 0 keeps the built-in P / L.  Variant
 * PK_VARIANT_STAGED sweeps whole pencils (n <= 256) two per CTA, staged in
 * shared memory by TMA bulk-tensor copies (P and L are then ignored); where
 * it cannot run (connected domains, stacked instances, WENO3, odd x extent or
 * guard width) the whole-pencil tile of variant 2 runs instead. */
#define PK_VARIANT_STAGED 7
int pk_set_tile(pk_handle h, int32_t dir, int32_t pencils, int32_t length, int32_t variant);

/* Arithmetic of the fused and batched sweeps (no counterpart in the
 * reference, whose arithmetic is gfortran -O2 SSE2 without FMA):
 *   PK_ARITH_BITEXACT (default): every operation in the reference's order and
 *     rounding; results equal the reference's bit for bit.
 *   PK_ARITH_FMA: multiply-add contraction and divisions by a common
 *     denominator replaced by one reciprocal (1/rho, 1/(gamma-1), 1/gamma,
 *     1/(S-S_M) and the other HLLD denominators, 1/ch); same branches and
 *     algorithm, rounding differs by a few units in the last place per
 *     operation, so a time step agrees with the bit-exact one to ~1e-15
 *     relative (tested to 1e-12 per step and 1e-9 after 100 steps).
 * The per-block stage path, the unsplit scheme and the adjoint kernels
 * always use the bit-exact arithmetic. */
enum { PK_ARITH_BITEXACT = 0, PK_ARITH_FMA = 1 };
int pk_set_arithmetic(pk_handle h, int32_t mode);

/* Sweep all blocks in one persistent launch over a work list of tiles (the
 * default whenever more than one block is registered; enable = 1 forces it for
 * a single block), with chunks of at most `length` cells and the given
 * launch-bound variant (-1 keeps the current one). */
int pk_set_batch(pk_handle h, int32_t enable, int32_t length, int32_t variant);

/* Refined domains (sweeps.F90:218-262, the finer level's boundary fluxes
 * replacing the coarser level's within each RK stage): one_launch = 1 sweeps
 * every level of a stage in one persistent launch whose work list holds the
 * levels' pencil tiles and the flux restriction between them, ordered so that
 * an item waits only for items listed before it; 0 (the default, about 3 %
 * faster on B200 for the 515-block three-level layout) launches level by
 * level with a restriction launch between.  Results are identical. */
int pk_set_refined_launch(pk_handle h, int32_t one_launch);

/* Replay the sweeps of a step (fluid_update) as one captured CUDA graph; the
 * step scalars (dt, chspeed, glmdamping factor) are read by the kernels from
 * device memory, so one capture serves every step. */
int pk_use_graph(pk_handle h, int32_t enable);

/* Launch-bound variant of the batched stage kernel that sweeps many blocks
 * stage by stage (refined or non-periodic connected domains): 0 = 320
 * threads x 1 CTA per SM (default), 1 = 128 x 3, 2 = 192 x 2, 3 = 384 x 1.  Used by the
 * tuning of the refined workload; WENO3 always runs variant 0. */
int pk_set_stage_variant(pk_handle h, int32_t variant);

/* ---- Independent instances in one launch ----
 * count independent, fully periodic problems of n[0] x n[1] x (n[2]/count)
 * cells stacked along z in the handle's single block (instance i owns the
 * interior z planes [i*n[2]/count, (i+1)*n[2]/count)).  Every sweep is one
 * launch over all instances; each instance wraps periodically inside its own
 * z range and advances with its own time state: its own CFL time step
 * (timestep.F90:158-228, reduction over its cells only), chspeed and
 * glmdamping factor.  The result of each instance is bit for bit that of a
 * handle holding that instance alone.  Needs RK2, every direction periodic,
 * no step retry, and n[2]/count in [nb, 256].  count = 1 returns to one
 * problem.  The reference runs such an ensemble as separate runs: no
 * counterpart in its code.  pk_time_step, pk_fluid_update, pk_run and the
 * pk_grad_* calls then act on all instances (the grad calls' dt arrays hold
 * count values per step, step-major); pk_get_time_state reports instance
 * 0 and pk_set_time_state sets every instance. */
int pk_set_instances(pk_handle h, int32_t count);
int pk_get_instance_state(pk_handle h, int32_t instance, pk_time_state* st);
int pk_set_instance_state(pk_handle h, int32_t instance, const pk_time_state* st);

/* ---- Connected blocks of one level (cg_list_bnd.F90:251-324) ----
 * pk_set_domain declares a level of ncells cells per direction (periodic or
 * not per direction); pk_block_place puts a block's first interior cell at
 * off on that grid.  From then on every guard refresh (pk_fill_guards, and
 * the one after each RK stage of pk_sweep) copies the neighbours' interior
 * cells into the guard cells that lie over them, after the blocks' own
 * boundary rules (outflow / reflecting) have filled the rest; the sweep runs
 * per RK stage (pk_solve_cg) for such a domain.  Overlapping blocks are
 * rejected at the first refresh. */
int pk_set_domain(pk_handle h, const int64_t ncells[3], const int32_t periodic[3]);
int pk_block_place(pk_handle h, int32_t id, const int64_t off[3]);

/* ---- Refined domains (several levels, refinement factor 2) ----
 * pk_block_place_level puts a block on level `level`, whose grid is the
 * base grid (pk_set_domain) refined `level` times, at offset off; the
 * block's cell size must be the base cell size / 2**level.  With blocks on
 * more than one level the domain must be periodic in every direction with
 * extent, level 0 must cover it, blocks of level >= 1 need even offsets and
 * extents and must lie two coarse cells inside their coarser level.  The
 * sweeps then run stage by stage as the reference's sweep does
 * (sweeps.F90:214-272): finest level first, each fine block's boundary
 * fluxes restricted (2 x 2 mean) into the coarser block's update through the
 * same face (fc_fluxes.F90:55-233, solve_cg_riemann.F90:353-362); after each
 * stage the guard cells of each level are copied from its own blocks, then
 * those over the coarser level only are prolonged from it, coarsest first:
 * fluids by injection, B and psi by the O_I2 interpolation
 * (cg_level_connected.F90:1150-1359, grid_container_prolong.F90:180-453).
 * pk_timestep_raw reduces over leaf cells only (timestep.F90:463). */
int pk_block_place_level(pk_handle h, int32_t id, int32_t level, const int64_t off[3]);

/* restrict_to_base (cg_level_connected.F90:1395-1409, restrict_1var
 * :1480-1721): every cell covered by a finer block takes the mean of its
 * 2**eff_dim children (u, B and psi), finest level first, as the reference
 * does before writing output or regridding; guard cells are not touched.
 * Synchronous.  No effect on a domain with one level. */
int pk_restrict(pk_handle h);

/* Fill the interior of block id (a refined level's) from the next coarser
 * level, as the reference's refinement update fills a new fine block
 * (cg_level_connected.F90:870-920 prolong, 1059-1093 prolong_1var): u and B
 * by injection (rank-4 arrays are prolonged at order 0 whatever their
 * registered order), psi at ord_mag_prolong.  With pk_restrict this lets a
 * host regrid: restrict, place the blocks of the new layout, fill the new
 * ones with pk_prolong_block, then pk_fill_guards.  The coarser level's guard
 * cells must be current (pk_fill_guards before the new blocks were placed).
 * Synchronous. */
int pk_prolong_block(pk_handle h, int32_t id);

/* ---- Refinement criteria (unified_ref_crit_var, URC_var.F90) ----
 * One criterion examines one plane of the block state (field: the plane
 * index, fluid components first in the reference's order, then B, then psi;
 * the reference's "dens" / "velx" / "ener" name every fluid's component of
 * that kind, i.e. one criterion per fluid).  A cell is flagged when any
 * criterion fires (cg%flag%set):
 *   PK_URC_THRESHOLD  field >= thr over the interior; none on levels >= aux
 *                     when aux > 0 (refine_on_threshold :297-330);
 *   PK_URC_GRAD       sum over directions of (p(+1) - p(-1))^2 >= thr^2
 *                     over the interior (refine_on_gradient :512-582);
 *   PK_URC_RELGRAD    the (+)-sum of |a - b| / (|a| + |b|) over the six
 *                     neighbours, squared, >= thr^2 (refine_on_relative_gradient
 *                     :589-708);
 *   PK_URC_LOECHNER   Loechner's second-derivative estimator with noise
 *                     filter aux >= thr, over the interior widened by two
 *                     cells along each direction (refine_on_second_derivative
 *                     :348-505; needs nb >= 4). */
#define PK_URC_THRESHOLD 0
#define PK_URC_GRAD 1
#define PK_URC_RELGRAD 2
#define PK_URC_LOECHNER 3

typedef struct pk_urc {
    int32_t method;     /* PK_URC_* */
    int32_t field;      /* plane of the block state */
    double thr;         /* ref_thr */
    double aux;         /* Loechner noise filter; threshold: first level left unmarked (> 0) */
} pk_urc;

/* scan_for_refinements' marking pass (refinement_update.F90:57-120): refresh
 * the guard cells (all_bnd), clear every block's flag map (flag%init) and
 * apply the criteria on every block with a leaf cell (urc_list%all_mark over
 * leaves).  flagged (host, one per block, may be null) receives 1 where a
 * leaf interior cell is flagged: the block may not be derefined
 * (sanitize_ref_flags :222-249).  The maps stay on the device for
 * pk_refine_map and pk_refine_candidates.  Synchronous. */
int pk_mark_refinement(pk_handle h, const pk_urc* crit, int32_t ncrit, int32_t* flagged);

/* Block id's flag map after pk_mark_refinement: one byte per guard-inclusive
 * cell, x fastest (cg%flag%map). */
int pk_refine_map(pk_handle h, int32_t id, uint8_t* map);

/* refinemap2SFC_list (grid_container_ref.F90:96-142) of block id: flags on
 * covered interior cells are dropped, then every bsize-sized block of the
 * next finer level whose parent cells inside this block's interior hold a
 * flag is listed by its offset on that level's grid (3 per candidate, x
 * outermost as the reference loops).  count receives the number found;
 * at most cap are written.  No candidates when bsize <= 0 along a direction
 * with extent (blocky AMR only). */
int pk_refine_candidates(pk_handle h, int32_t id, const int32_t bsize[3], int64_t* offsets, int32_t cap,
                         int32_t* count);

/* ---- Domains spanning ranks (one process per GPU) ----
 * The reference exchanges guard cells between MPI ranks in the same
 * internal_boundaries pass (cg_list_bnd.F90:251-324, MPI isend/irecv of the
 * segment buffers) and reduces dt over ranks (timestep.F90:173).  Here the
 * library plans and packs, the host moves the bytes (NCCL, MPI, ...):
 *   pk_block_remote declares a block of the same level held by rank owner
 *   (every rank declares all blocks it does not hold);
 *   pk_halo_peers lists the ranks this one exchanges with, pk_halo_sizes the
 *   doubles sent to / received from one of them per exchange;
 *   pk_halo_pack fills a device buffer with the cells a peer needs,
 *   pk_halo_unpack writes a peer's buffer into the guard cells (both
 *   synchronous on the handle's stream);
 *   pk_set_comm installs host callbacks: halo(ctx, dir) runs after every
 *   local guard exchange (dir = the sweep direction 0..2, or -1) and must
 *   pack, move and unpack for all peers; reduce(ctx, x, op) returns the
 *   minimum (op 0) or maximum (op 1) of x over ranks and is used for dt and
 *   c_all in pk_time_step, for chspeed (grid: minimum, hdc.F90:138; gas:
 *   maximum) and the glmdamping factor (minimum, hdc.F90:333) in each
 *   fluid update, and for the negatives flag of the step retry (maximum);
 *   every rank makes these calls in the same order.  With callbacks set,
 *   pk_run does not use graphs.
 * Both sides order a peer's cells alike (by positions on the level's grid). */
typedef void (*pk_halo_fn)(void* ctx, int32_t dir);
typedef double (*pk_reduce_fn)(void* ctx, double x, int32_t op);
int pk_block_remote(pk_handle h, int32_t owner, const int32_t n[3], const int64_t off[3]);
int pk_halo_peers(pk_handle h, int32_t* peers, int32_t max_peers, int32_t* count);
int pk_halo_sizes(pk_handle h, int32_t peer, int64_t* send_doubles, int64_t* recv_doubles);
int pk_halo_pack(pk_handle h, int32_t peer, double* sendbuf_dev);
int pk_halo_unpack(pk_handle h, int32_t peer, const double* recvbuf_dev);
int pk_set_comm(pk_handle h, pk_halo_fn halo, pk_reduce_fn reduce, void* ctx);
/* The same per sweep direction (no counterpart in the reference, which
 * exchanges every guard cell before every sweep): dir 0..2 restricts a
 * peer's traffic to the face boxes of the guard region along dir -- all a
 * fused sweep along dir reads -- and dir = -1 is the whole halo as above.
 * For z slabs of a periodic domain, x and y sweeps then move nothing between
 * ranks.  Unlike pk_halo_pack / pk_halo_unpack these two do not wait: the
 * copies are ordered on the handle's stream (pk_stream), so a transport that
 * enqueues its sends after the pack and makes that stream wait for its
 * receives (NCCL on the same stream) needs no host synchronisation; the
 * buffers must stay valid until the stream has passed them. */
int pk_halo_sizes_dir(pk_handle h, int32_t peer, int32_t dir, int64_t* send_doubles, int64_t* recv_doubles);
int pk_halo_pack_dir(pk_handle h, int32_t peer, int32_t dir, double* sendbuf_dev);
int pk_halo_unpack_dir(pk_handle h, int32_t peer, int32_t dir, const double* recvbuf_dev);

/* ---- Differentiable path (one periodic block, one fluid, RK2) ----
 * Not in the reference, which has no derivatives: the adjoint (reverse
 * mode) of the sweep path at a fixed sequence of time steps. */

/* Device-to-device state transfer (structure of arrays with guard cells,
 * nplanes x ext_x*ext_y*ext_z doubles; guards are refreshed on upload). */
int pk_upload_device(pk_handle h, int32_t id, const double* soa_dev);
int pk_download_device(pk_handle h, int32_t id, double* soa_dev);

/* The adjoint state dL/dU in the same layout, from/to host (on_device = 0) or
 * device memory.  Guard values are ignored on input and zero on output. */
int pk_adjoint_set(pk_handle h, int32_t id, const double* lam, int32_t on_device);
int pk_adjoint_get(pk_handle h, int32_t id, double* lam, int32_t on_device);

/* lam <- (d sweep(cdim)/dU)^T lam at the current state (one fused sweep). */
int pk_adjoint_sweep(pk_handle h, int32_t cdim, double dt, double chspeed);

/* Advance nsteps steps like pk_run, recording dt / chspeed / glmdamping per
 * step and checkpointing the state every `every` steps.  dt_in (nsteps
 * values, or NULL for the CFL time step) replays a prescribed sequence;
 * dt_out (or NULL) receives the steps taken. */
int pk_grad_forward(pk_handle h, int32_t nsteps, int32_t every, const double* dt_in, double* dt_out);

/* Given lam = dL/d(final state) (pk_adjoint_set), leave lam = dL/d(state at
 * the start of pk_grad_forward): each checkpointed segment is recomputed once
 * and its steps' sweeps are reversed with the adjoint sweep kernel. */
int pk_grad_backward(pk_handle h);
int pk_grad_release(pk_handle h);

/* Tile of the adjoint sweep kernels along dir (0..2, -1: all): owned cells
 * per pencil (0: default) and launch-bound variant (-1: default; 0..4 tiled
 * variants; 5 the TMA-staged whole-pencil kernels, which fall back to variant
 * 0 where the block does not allow them). */
int pk_set_adjoint_tile(pk_handle h, int32_t dir, int32_t length, int32_t variant);

/* ---- Measurement utility ----
 * No counterpart in the reference.  The FP64 fused-multiply-add throughput
 * of the current device in TFLOP/s (2 flops per DFMA), measured with a
 * latency-free DFMA kernel: the denominator of the sweep kernels' FP64
 * roofline.  Allocates 2 KiB of device memory for the call's duration. */
int pk_fp64_peak(double* tflops);

/* ---- Raw CFL time step without allocation ----
 * No counterpart in the reference.  For host codes that cannot let this
 * library allocate device memory (all of it is reserved for their own pool,
 * or a cudaMalloc would synchronise the device inside their step loop) and so
 * cannot create a handle: the same result as pk_timestep_raw over nblocks
 * blocks whose states the caller holds in device memory, each in the
 * handle's layout (component planes u, then bx, by, bz, psi when magnetic;
 * each plane ext_x*ext_y*ext_z doubles with ext = n + 2*nb where n > 1,
 * else 1).  n and dl hold 3 values per block; states holds nblocks device
 * pointers of the current device; stream may be NULL (the legacy default
 * stream) or a stream of the current device.  The call is synchronous (it
 * reads the result back and waits for the stream) and allocates nothing: its
 * reduction slots are a fixed 6 KiB device array, kept by every GPU that
 * loads the library until exit and shared by all calls, so calls that
 * overlap on one GPU race.  At most PK_NOALLOC_MAX_BLOCKS blocks per call
 * (PK_E_ARG beyond).  A state that is not device memory of the current
 * device, or a stream of another device, gives PK_E_ARG before anything is
 * launched; a call while the stream is capturing gives PK_E_STATE.  The first
 * call on a device looks up the array's address there.  err (errlen bytes,
 * or NULL) receives a message. */
#define PK_NOALLOC_MAX_BLOCKS 64
int pk_timestep_raw_noalloc(const pk_config* cfg, int32_t nblocks, const int32_t* n, const double* dl,
                            const double* const* states, void* stream, double* dt_out, double* c_all_out,
                            char* err, int32_t errlen);

/* Launch-bound variants of the fused sweep: count, CTA size and CTAs per SM
 * each was compiled for (arrays of at least 16 entries). */
int pk_tile_variants(int32_t* n, int32_t* threads, int32_t* ctas_per_sm);

/* CUDA stream of the handle (cudaStream_t), for callers that interleave work. */
void* pk_stream(pk_handle h);

/* Kernel accounting.  With profiling on, every sweep kernel is bracketed by a
 * pair of CUDA events on the handle's stream.  pk_profile_read waits for the
 * stream and returns the number of this library's kernel launches since the
 * handle was created, the number of sweep launches timed since the last read
 * and their summed device time in milliseconds. */
int pk_profile_enable(pk_handle h, int32_t on);
int pk_profile_read(pk_handle h, int64_t* launches, int64_t* sweep_launches, double* sweep_ms);

#ifdef __cplusplus
}
#endif
#endif
