/*
 * pk_oracle.h -- TEST INFRASTRUCTURE, NOT PRODUCT CODE.
 *
 * CPU restatement of PIERNIK's split Riemann sweep (RIEMANN_SPLIT solver),
 * used only by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg, as the checker the CUDA library is compared against.
 *
 * Parity status: pinned by the reference's known answers.  The reference is
 * Fortran 2008 and no Fortran compiler exists in this environment; its gold
 * tests regenerate outputs from upstream git.  Its CPAW artifact test
 * (Makefile CPAW target, problems/cpaw/problem.par:1-13) tabulates the L2
 * error of B after one wave period at eight resolutions; the restatement,
 * run through the unsplit scheme (which shares utoq, the limiters, HLLD with
 * GLM, the floors, the CFL reduction and the GLM scalars with the split
 * sweep), reproduces every one to the 8 printed decimals (tests/test_cpaw.py).
 * The split-only structure (sweep order, per-sweep RK stages) follows the
 * reference sources operation by operation (evaluation order, Fortran
 * intrinsics spacing/sign/min/max, the -0.0 normalisation done by
 * internal_sources) and is cross-checked by physics properties in tests/
 * (conservation, axis-permutation symmetry) and exact solutions (Sod's shock
 * tube for HLLC with every limiter, stationary contacts and tangential
 * discontinuities for HLLC / HLLD, dust advection, second-order convergence
 * of the split sweep on the CPAW wave).
 *
 * Layout mirrors the reference's named arrays with guard cells:
 *   u  (nvar, i, j, k)  -> u[((k*NY + j)*NX + i)*nvar + v]   (cg%u, cg%w(uh))
 *   b  (3,    i, j, k)  -> b[((k*NY + j)*NX + i)*3 + d]      (cg%b, magh)
 *   psi(i, j, k)        -> psi[(k*NY + j)*NX + i]            (cg%q(psi), psih)
 * where NX = n[0] + 2*g[0] and g[d] = nb when the direction exists, else 0
 * (src/grid/grid_container_base.F90 extents lhn/ijkse).
 */
#ifndef PK_ORACLE_H
#define PK_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

enum { O_ION = 0, O_NEU = 1, O_DST = 2 };
enum { O_LIM_VANLEER = 0, O_LIM_MINMOD = 1, O_LIM_MONCEN = 2, O_LIM_SUPERBEE = 3 };
enum { O_BND_PER = 0, O_BND_OUT = 1, O_BND_REF = 2 };

#define O_MAXFL 3

typedef struct o_cfg {
    int nfluids;                 /* fluids in flind order: ionized, neutral, dust */
    int kind[O_MAXFL];           /* O_ION / O_NEU / O_DST */
    double gamma[O_MAXFL];       /* adiabatic index; dust uses gamma < 0 */
    int magnetic;                /* 1: B + GLM psi registered (divB_0 = HDC) */
    int limiter, limiter_b;      /* flimiter / blimiter */
    int use_smalld, use_smallei;
    int disallow_negatives;
    double smalld, smallei;
    double cfl, cfl_glm, glm_alpha;
    int ch_grid;
    int integration_order;       /* 1 (EULER) or 2 (RK2) */
    double dt_initial, dt_max_grow, dt_min, dt_max, tend;
    int skip_sweep[3];
    int cflcontrol;              /* O_CFL_NONE / O_CFL_WARN / O_CFL_REDO (global.F90:218, timestep.F90:73-90) */
    double cfl_max, dt_shrink;   /* global.F90:233,245 (cfl_max sanitized as :304 on use) */
    int max_redostep_attempts;   /* global.F90:258 */
    int interpolation;           /* 0 linear, 1 weno3 (interpol_str, global.F90:220) */
    double w_epsilon;            /* global.F90:255 */
    int solver;                  /* 0 RIEMANN_SPLIT, 1 RIEMANN_UNSPLIT (solver_str, global.F90:423-437) */
    int use_eglm;                /* E-GLM sources after each triple of sweeps (global.F90:109,252; hdc.F90:355-457) */
} o_cfg;

#define O_CFL_NONE 0
#define O_CFL_WARN 1
#define O_CFL_REDO 2
#define O_CFL_FLEX 3             /* timestep.F90:81-84: redo with flexible_shrink */
#define O_CFL_AUTO 4             /* timestep.F90:85-86: cfl_auto */

/* Fine/coarse flux hooks of one block along one direction (fluxtypes.F90
 * ext_fluxes, set by grid_container_fcflx.F90:148-259).  Pencils are
 * numbered (i1 - g[o1]) + n[o1] * (i2 - g[o2]) with (o1, o2) the reference's
 * ORTHO1 / ORTHO2 of the direction.  A flux vector is the pencil's nvar flux
 * columns (in the pencil's column order) followed, when magnetic, by the 4
 * mag_flx columns. */
typedef struct o_eflx {
    int *in_face[2];             /* per pencil: 0-based face (between pencil cells k and k+1) whose
                                    flux is replaced, -1 none; [0] li, [1] ri */
    double *in_flx[2];           /* per pencil: the replacing flux vector */
    int *out_on[2];              /* per pencil: record the face before the first ([0], lo) or
                                    after the last ([1], ro) interior cell */
    double *out_flx[2];          /* per pencil: the recorded flux vector */
} o_eflx;

typedef struct o_block {
    int n[3];                    /* interior cells per direction */
    int nb;                      /* guard cells (dom%nb) */
    double dl[3];                /* cell sizes */
    int bnd[3][2];               /* O_BND_* per side */
    double *u, *uh;              /* nvar components */
    double *b, *bh;              /* 3 components (NULL when !magnetic) */
    double *psi, *psih;          /* (NULL when !magnetic) */
    int dn_negative, ei_negative;
    double *uh_retry;            /* step-retry backup of u, b, psi (nvar+4 planes of the guard-inclusive block), or NULL */
    const unsigned char *leaf;   /* interior cells not covered by a finer block (i fastest), or NULL: all */
    const o_eflx *eflx[3];       /* fine/coarse flux hooks per direction, or NULL */
} o_block;

typedef struct o_state {         /* the reference's global time-step state */
    double t, dt, dt_old, c_all, chspeed;
    int nstep;
    /* step retry (timestep_retry.F90, timestep.F90:247-360) */
    double dt_full, c_all_old, dt_cur_shrink, stepcfl, t_saved;
    int nstep_saved, tstep_attempt, repeat, redone;
    double cfl_c;                /* cfl_auto's factor (timestep_pub.F90:42, initially one) */
} o_state;

int    o_nvar(const o_cfg *cfg);
double o_cfl_max(const o_cfg *cfg);
int    o_run_fixed(const o_cfg *cfg, o_block *blk, o_state *st, const double *dts, int nsteps);
void   o_extents(const o_block *blk, int ext[3], int g[3]);

/* one stage of solve_cg_riemann on one block (solve_cg_riemann.F90:68-233,241-307) */
int    o_solve_cg(const o_cfg *cfg, o_block *blk, int ddim, int istep, double dt, double ch);
/* guardcell refresh of u, b, psi (sweeps.F90:66-107 for a single block) */
void   o_fill_guards(const o_cfg *cfg, o_block *blk);
/* sweep(cdim): RK stages + boundary update (sweeps.F90:114-279) */
int    o_sweep(const o_cfg *cfg, o_block *blk, int cdim, double dt, double ch);
/* glmdamping factor and application (hdc.F90:289-349) */
double o_glm_fac(const o_cfg *cfg, const o_block *blk, double dt, double ch);
/* the unsplit scheme (src/scheme/unsplit_schemes): one stage (istep 1: first),
 * the sweep of all stages with boundary updates, fluid_update_unsplit */
int    o_unsplit_stage(const o_cfg *cfg, o_block *blk, int istep, double dt, double ch);
int    o_unsplit_sweep(const o_cfg *cfg, o_block *blk, double dt, double ch);
int    o_fluid_update_unsplit(const o_cfg *cfg, o_block *blk, o_state *st);
void   o_glm_apply(const o_cfg *cfg, o_block *blk, double fac);
/* E-GLM sources of one block for dt (hdc.F90:eglm), then its boundary update */
void   o_eglm(const o_cfg *cfg, o_block *blk, double dt);
/* update_chspeed with ch_grid (hdc.F90:90-140) */
double o_chspeed(const o_cfg *cfg, const o_block *blk, double dt);
/* timestep_fluid over all fluids, before clamps (timestep.F90:431-495) */
void   o_timestep_raw(const o_cfg *cfg, const o_block *blk, double *dt, double *c_all);
/* time_step(dt, flind, .true.) including the sanity clamps (timestep.F90:112-240) */
int    o_time_step(const o_cfg *cfg, const o_block *blk, o_state *st);   /* 3: dt < dt_min */
/* fluid_update_full (fluidupdate.F90:99-136) */
int    o_fluid_update(const o_cfg *cfg, o_block *blk, o_state *st);
/* main-loop body repeated nsteps times (piernik.F90:125-213 without I/O) */
int    o_run(const o_cfg *cfg, o_block *blk, o_state *st, int nsteps);
/* the same over several independent blocks sharing one dt (the leaves list) */
int    o_time_step_multi(const o_cfg *cfg, o_block *const *blks, int nb, o_state *st);
int    o_fluid_update_multi(const o_cfg *cfg, o_block *const *blks, int nb, o_state *st);
int    o_run_multi(const o_cfg *cfg, o_block *const *blks, int nb, o_state *st, int nsteps);
void   o_set_threads(int n);
int    o_get_threads(void);

#ifdef __cplusplus
}
#endif
#endif
