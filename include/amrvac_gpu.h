/*
 * amrvac_gpu.h — C ABI of the B200 finite-volume block update for MPI-AMRVAC.
 *
 * The library replaces the per-block loops of the reference's hot path:
 *   - advect1's OpenMP block loop calling advect1_grid -> finite_volume
 *     (src/mod_advance.t:611-666, src/mod_finite_volume.t:116-339),
 *   - setdt's block loop calling getdt_courant (src/mod_dt.t:10-155, 160-287),
 *   - getbc's same-resolution fill and physical cont/symm/asymm boundaries
 *     (src/mod_ghostcells_update.t:350-615, 812-852),
 *   - the SSP-RK stage algebra of advect (src/mod_advance.t:249-267).
 * Physics follows the reference plugin interface (src/physics/mod_physics.t:
 * phys_to_primitive/phys_to_conserved, phys_get_flux, phys_get_cbounds,
 * phys_modify_wLR, phys_add_source, phys_handle_small_values).
 *
 * Conventions
 *   - All entry points return int: 0 = OK, negative = configuration / usage
 *     error (AMRVAC_E_*), positive = runtime status bits (AMRVAC_ST_*).
 *   - Host arrays are the Fortran block arrays w(ixG^S,1:nw) (column-major,
 *     x fastest, variable slowest, ghost cells included), one block after
 *     another.  They are borrowed only for the duration of the call.
 *   - The library owns all device memory.  One CUDA stream per context.
 *     Calls on one context are not reentrant; call from one host thread.
 *   - Block ids are 0-based.  neighbor[] holds, per block, 3^ndim entries
 *     ordered with the x offset fastest ((di+1) + 3(dj+1) + 9(dk+1)); -1
 *     marks a physical boundary (the reference's neighbor_type==1).
 */
#ifndef AMRVAC_GPU_H
#define AMRVAC_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* configuration errors */
#define AMRVAC_E_ARG          (-1)  /* bad argument / null pointer */
#define AMRVAC_E_UNSUPPORTED  (-2)  /* option outside this library's scope */
#define AMRVAC_E_CUDA         (-3)  /* CUDA runtime error (see amrvac_gpu_last_error) */
#define AMRVAC_E_STATE        (-4)  /* call order (e.g. no blocks set) */
/* runtime status bits (OR-ed, sticky until amrvac_gpu_clear_status) */
#define AMRVAC_ST_SMALL_VALUE  1u   /* small density/pressure (the reference's crash) */
#define AMRVAC_ST_NAN          2u
#define AMRVAC_ST_DT_TOO_SMALL 4u   /* dt < dtmin (src/mod_dt.t:55-60) */
#define AMRVAC_ST_BOUNDS       8u   /* inconsistent neighbour table (read clamped) */
#define AMRVAC_ST_TIMEOUT     16u   /* an asynchronous plane copy of the stage kernel did not complete in time */

/* flux_scheme (src/mod_finite_volume.t method ids are private; names match) */
#define AMRVAC_FS_TVDLF 1
#define AMRVAC_FS_HLL   2
#define AMRVAC_FS_HLLC  3
#define AMRVAC_FS_HLLD  4
#define AMRVAC_FS_TVDMU 5  /* TVD-MUSCL (HD; with dimsplit, as the reference runs it) */
/* limiter ids: src/limiter/mod_limiter.t:14-24 */
#define AMRVAC_LIM_MINMOD   1
#define AMRVAC_LIM_WOODWARD 2
#define AMRVAC_LIM_MCBETA   3
#define AMRVAC_LIM_SUPERBEE 4
#define AMRVAC_LIM_VANLEER  5
#define AMRVAC_LIM_ALBADA   6
#define AMRVAC_LIM_KOREN    7
#define AMRVAC_LIM_CADA     8
#define AMRVAC_LIM_CADA3    9
#define AMRVAC_LIM_SCHMID   10  /* schmid2 (a2max = schmid_rad), schmid1 with schmid_global */
#define AMRVAC_LIM_VENK     11  /* Venkatakrishnan */
#define AMRVAC_LIM_MP5      13  /* fifth order, uniform grids, nghostcells >= 3 */
#define AMRVAC_LIM_WENO3    14  /* third-order WENO */
#define AMRVAC_LIM_WENOYC3  15  /* third-order WENO-YC */
#define AMRVAC_LIM_WENO5    16  /* WENO-JS, likewise */
#define AMRVAC_LIM_WENOZ5   18  /* WENO-Z, likewise */
#define AMRVAC_LIM_WENOZP5  20  /* WENO-Z+, likewise */
/* typeboundspeed: src/io/mod_input_output.t:1632-1641 */
#define AMRVAC_BS_EINFELDT      1
#define AMRVAC_BS_CMAXMEAN      2
#define AMRVAC_BS_CMAXLEFTRIGHT 3
/* typedivbfix: src/mhd/mod_mhd_phys.t divb_* ids */
#define AMRVAC_DIVB_NONE  0
#define AMRVAC_DIVB_GLM   1
#define AMRVAC_DIVB_LINDE 4
/* typecourant: mod_global_parameters type_maxsum/type_summax/type_minimum */
#define AMRVAC_COURANT_MAXSUM  1
#define AMRVAC_COURANT_SUMMAX  2
#define AMRVAC_COURANT_MINIMUM 3
/* typeboundary per side and variable: subset of mod_boundary_conditions bc_* */
#define AMRVAC_BC_PERIODIC 0
#define AMRVAC_BC_CONT     1
#define AMRVAC_BC_SYMM     2
#define AMRVAC_BC_ASYMM    3
/* time_stepper / time_integrator (src/mod_advance.t:56-567) */
#define AMRVAC_TS_ONESTEP   1   /* Forward_Euler */
#define AMRVAC_TS_TWOSTEP   2   /* Predictor_Corrector (default) or ssprk2 (Heun) */
#define AMRVAC_TS_THREESTEP 3   /* ssprk3, ssprk_order 3 or 2 */
#define AMRVAC_TS_FOURSTEP  4   /* ssprk4 (ssprk_order 3: SSPRK(4,3), 2: SSP(4,2)) or rk4 */
#define AMRVAC_TS_FIVESTEP  5   /* ssprk5: SSPRK(5,4) (ssprk_order 3: Gottlieb 2005, 2: Spiteri-Ruuth) */
#define AMRVAC_TI_DEFAULT   0   /* time_integrator: the stepper's default (twostep:
                                   Predictor_Corrector, threestep: ssprk3, fourstep: ssprk4) */
#define AMRVAC_TI_RK4       1   /* fourstep: the classical RK(4,4) */
#define AMRVAC_TI_SSPRK2    2   /* twostep: ssprk2 (Heun) */

#define AMRVAC_MAX_NW 16

/* Mirrors the par-file namelist variables the path reads (methodlist,
 * boundlist, meshlist, paramlist, hd_list / mhd_list). */
typedef struct amrvac_cfg {
  int ndim;                 /* 2 or 3 (1-D: see amrvac_gpu_create) */
  int ndir;                 /* vector components (2.5D: ndim=2, ndir=3) */
  int physics;              /* 0 = hd, 1 = mhd */
  int block_nx[3];          /* block_nx^D, the same in every direction: 8, 10, 12, 16 or 32 */
  int nghostcells;          /* ghost width of the host arrays (2) */
  double gamma;             /* hd_gamma / mhd_gamma */
  int flux_scheme;          /* AMRVAC_FS_* (one for all levels) */
  int limiter;              /* AMRVAC_LIM_* */
  int typeboundspeed;       /* AMRVAC_BS_* */
  int typedivbfix;          /* AMRVAC_DIVB_* (mhd) */
  double mhd_glm_alpha;     /* 0.5 */
  int mhd_glm_extended;     /* 1 */
  double divbdiff;          /* 0.8 (Linde) */
  double courantpar;        /* 0.8 */
  int type_courant;         /* AMRVAC_COURANT_* */
  double cada3_radius;      /* 0.1 */
  double tvdlfeps;          /* 1.0 */
  int fix_small_values;     /* 0 */
  int check_small_values;   /* 1 */
  int small_values_method;  /* 0 = error, 1 = replace, 2 = average */
  double small_density, small_pressure;
  int time_stepper;         /* AMRVAC_TS_* */
  int ssprk_order;          /* 3 */
  double dtmin;             /* 1e-10 */
  int typeboundary[6][AMRVAC_MAX_NW]; /* [min1,max1,min2,max2,min3,max3][iw] */
  int zchunk;               /* work distribution: 0 = persistent plane ranges
                               (default), 16/8/4 = z-planes per CTA in 3-D */
  int precision;            /* 0 = plain FP64; 1 = mixed: FP32 reconstruction, wave
                               speeds, fluxes, Riemann solver; FP64 conserved state,
                               pressure recovery, accumulation, sources, small values */
  int slowsteps;            /* setdt ramp (src/mod_dt.t:64-67): during the first
                               slowsteps steps after amrvac_gpu_set_time, dt is
                               scaled by 1 - (1 - n/slowsteps)^2 (n = 1, 2, ...);
                               <= 0: off (default -1) */
  int time_integrator;      /* AMRVAC_TI_* (src/mod_advance.t:454-512) */
  int dimsplit;             /* 0 unsplit (default); 1 dimensionally split with
                               typedimsplit 'xyyx' (the order reverses on odd
                               steps), 2 'xy' (src/mod_advance.t:23-45) */
  double schmid_rad[3];     /* schmid limiter radii per direction (default 1) */
  int schmid_global;        /* 1: schmid1, a2max from the domain every setdt
                               (need_global_a2max) instead of schmid_rad; the
                               getdt phase reduces it, so amrvac_gpu_advect1 /
                               advect1_dim / step_dt return AMRVAC_E_STATE until
                               an amrvac_gpu_getdt has run on the current state
                               (after an upload, set_blocks or regrid) */
  int small_values_daverage; /* small_values_daverage (src/mod_small_values.t:12):
                               largest cube half-width of method 'average'
                               (default 1) */
} amrvac_cfg;

typedef struct amrvac_ctx amrvac_ctx;

/* Fill *cfg with the reference defaults (src/io/mod_input_output.t:284-480). */
void amrvac_gpu_default_cfg(amrvac_cfg *cfg);
/* Number of conserved variables (nwflux) implied by cfg. */
int amrvac_gpu_nw(const amrvac_cfg *cfg);

/* Create a context on the current CUDA device.  Refuses unsupported options
 * (AMRVAC_E_UNSUPPORTED), e.g.: 1-D, ndir < ndim, block_nx other than 8, 10,
 * 12, 16, 32 (and, other than 16, MP5/WENO5),
 * small_values_method 'average' with dimsplit, Linde, the MUSCL-Hancock
 * predictor or a limiter outside dwlimiter2; the text comes from
 * amrvac_gpu_last_error().  The configuration has no geometry field: blocks
 * are Cartesian. */
int amrvac_gpu_create(const amrvac_cfg *cfg, amrvac_ctx **ctx);
int amrvac_gpu_destroy(amrvac_ctx *ctx);

/* Define the block set (replaces the host's ps(:) list for the path).
 * dx: [nblocks][ndim] cell sizes (rnode(rpdx^D_,igrid)); neighbor as above. */
int amrvac_gpu_set_blocks(amrvac_ctx *ctx, int nblocks, const double *dx, const int *neighbor);
/* Convenience: uniform level-1 grid, blocks ordered x fastest; periodicity
 * from cfg->typeboundary. */
int amrvac_gpu_set_uniform_grid(amrvac_ctx *ctx, const int *domain_nx, const double *xprobmin,
                                const double *xprobmax);
int amrvac_gpu_nblocks(const amrvac_ctx *ctx);
/* Static multi-level grid (replaces the forest and neighbour search of
 * src/amr/mod_forest.t and src/amr/mod_amr_neighbors.t for a fixed tree):
 * leaf[4*b] = level (1-based), ig0, ig1, ig2 (block index at that level);
 * nbase root blocks per direction over [xprobmin, xprobmax]; the boundary
 * kinds of cfg->typeboundary (a dimension periodic on both sides or
 * neither), ndim 2 or 3, nghostcells 2, 2:1 balanced across faces, edges
 * and corners.  Blocks are numbered in the order given.  Afterwards every
 * stage fills the level-jump ghost cells as the reference's multi-level getbc
 * does (restriction, and prolongation by interpolation_linear,
 * src/mod_ghostcells_update.t:350-578, 1381-1525) and applies the flux fix
 * (store_flux / fix_conserve, src/mod_fix_conserve.t:465-648); download
 * returns those ghost cells too.  Replaces any previous block set. */
int amrvac_gpu_set_amr_grid(amrvac_ctx *ctx, int nleaf, const int *leaf, const int *nbase, const double *xprobmin,
                            const double *xprobmax);
/* Regrid in place (replaces amr_coarsen_refine, src/amr/mod_coarsen_refine.t:
 * 20-182, for a tree the host has decided): the new leaves as for
 * amrvac_gpu_set_amr_grid (same domain and root blocks), and per new leaf
 * op[9*b]: {0, old} copy of an old leaf; {1, old parent, child bits} a child
 * of a refined old leaf, by prolong_2nd (src/amr/mod_refine.t:81-167) from
 * the parent and its getbc ghost values; {2, old children in child-bit
 * order} a coarsened parent, by coarsen_grid (src/amr/mod_coarsen.t:12-79).
 * Ops that do not match the old and new trees are refused.  Register 0
 * carries the state over; registers 1 and 2 are scratch afterwards. */
int amrvac_gpu_amr_regrid(amrvac_ctx *ctx, int nleaf, const int *leaf, const int *op);
/* resettree (src/amr/mod_amr_grid.t:45-73): errest with the Löhner
 * estimator on register 0 (arguments as for amrvac_gpu_lohner, levels taken
 * from the current tree), the tree decision below, and amrvac_gpu_amr_regrid.
 * *changed (may be NULL) = 1 when the tree changed. */
int amrvac_gpu_amr_resettree(amrvac_ctx *ctx, const double *weight, const int *logflag, int refine_max_level,
                             const double *refine_threshold, const double *derefine_ratio,
                             const double *amr_wavefilter, int *changed);
/* The current leaves, 4 ints each (level, ig0, ig1, ig2) in block order, if
 * leaf is not NULL; returns their number (AMRVAC_E_STATE without a grid). */
int amrvac_gpu_amr_leaves(const amrvac_ctx *ctx, int *leaf);
/* The tree decision of amr_coarsen_refine with proper_nesting
 * (src/amr/mod_coarsen_refine.t:20-319), host only: from the leaves (on a
 * domain periodic in the dimensions flagged in periodic) and the
 * per-leaf refine / coarsen flags, the new leaves (sorted by level, ig0, ig1,
 * ig2) and their ops for amrvac_gpu_amr_regrid.  cap = capacity of leaf_new
 * (4 ints per leaf) and op (9 ints per leaf) in leaves; *nnew is set even
 * when it exceeds cap (then AMRVAC_E_ARG). */
int amrvac_amr_plan(int ndim, const int *nbase, const int *periodic /* [ndim], NULL: all periodic */,
                    int max_level, int nleaf, const int *leaf, const unsigned char *refine,
                    const unsigned char *coarsen, int cap, int *nnew, int *leaf_new, int *op);
/* Blocks next to a level jump (0 on a single-level grid). */
int amrvac_gpu_amr_slots(const amrvac_ctx *ctx);
/* Average device time of the level-jump ghost pass (register 0) and of the
 * flux fix (applied to register 2, which it changes) over reps launches. */
int amrvac_gpu_amr_kernel_ms(amrvac_ctx *ctx, int reps, double *ghost_ms, double *fix_ms);

/* Copy n blocks starting at `first` between host Fortran arrays and register
 * reg (0 = ps, 1 = ps1, 2 = ps2).  Upload reads interior cells only; download
 * fills ghost cells as getbc would (same-resolution copy + physical BC). */
int amrvac_gpu_upload(amrvac_ctx *ctx, int reg, int first, int n, const double *w);
int amrvac_gpu_download(amrvac_ctx *ctx, int reg, int first, int n, double *w);

/* getdt_courant over all blocks of register reg: CFL dt (before any output /
 * time_max clipping) and cmax_global.  Synchronous. */
int amrvac_gpu_getdt(amrvac_ctx *ctx, int reg, double *dt, double *cmax_global);

/* One explicit stage (advect1 on all blocks):
 *   w[reg_new] = a_base*w[reg_base] + b_in*w[reg_ct]  (a_base==0: = w[reg_ct])
 *   then finite_volume(qdt=dtfactor*dt) with wCT = w[reg_ct] and sources.
 * Uses cmax_global from the last getdt / set_cmax_global, and with schmid1
 * the a2max_global of the last getdt (AMRVAC_E_STATE if none has run on the
 * current state).  Asynchronous. */
int amrvac_gpu_advect1(amrvac_ctx *ctx, int reg_ct, int reg_new, int reg_base, double a_base,
                       double b_in, double dtfactor, double dt);
/* The same stage restricted to direction idim (1..ndim; 0: all), as advect1
 * with idim^LIM = idim, idim in a dimensionally split step
 * (src/mod_advance.t:23-45, 611-666): that direction's fluxes, its flux fix
 * on multi-level grids, and the divB sources with qdt / ndim.  Synchronous. */
int amrvac_gpu_advect1_dim(amrvac_ctx *ctx, int reg_ct, int reg_new, int reg_base, double a_base,
                           double b_in, double dtfactor, double dt, int idim);
int amrvac_gpu_set_cmax_global(amrvac_ctx *ctx, double cmax_global);

/* Time control for amrvac_gpu_step: current time, time_max (final_dt_reduction)
 * and one output interval dtsave (0 = none), as in setdt (src/mod_dt.t:69-99). */
int amrvac_gpu_set_time(amrvac_ctx *ctx, double global_time, double time_max, double dtsave);
/* One full time step on register 0: setdt on the device, the configured RK
 * stages, global_time += dt.  Asynchronous; no host round trip. */
int amrvac_gpu_step(amrvac_ctx *ctx);
/* nsteps steps, captured once into a CUDA graph and replayed. */
int amrvac_gpu_run(amrvac_ctx *ctx, int nsteps);
/* nsteps steps launched directly (no graph) with CUDA events recorded on the
 * context stream around every kernel; returns the whole elapsed time and the
 * summed durations of the stage kernels and of the getdt kernels (ms).
 * Synchronises.  Used for live per-kernel timing inside a benchmark. */
int amrvac_gpu_run_timed(amrvac_ctx *ctx, int nsteps, double *total_ms, double *stage_ms, double *getdt_ms);
/* Measured FP64 FMA throughput of the current device (TFLOP/s, 2 flops per
 * FMA) from an in-register FMA-chain kernel; the FP64 roofline denominator. */
int amrvac_gpu_fp64_peak(double *tflops);
/* Diagnostic of the bounded wait of the stage kernel's asynchronous plane
 * staging (no counterpart in the reference): one CTA waits on an mbarrier
 * phase that nothing completes, gives up after `spins` polls (1 ..
 * 4194304) and sets AMRVAC_ST_TIMEOUT in *flags (host) — the path a stage
 * takes when a bulk copy does not arrive; the device stays usable.
 * Synchronous. */
int amrvac_gpu_wait_probe(int spins, uint32_t *flags);
/* Autotuner (no counterpart in the reference, whose block loop has no launch
 * shape): times one stage (ps -> ps1, the state in ps is left unchanged) for
 * each stage-kernel variant of the scheme with each work distribution —
 * 0: persistent CTAs (one wave), each marching a contiguous range of
 * z-planes across blocks; block_nx, block_nx/2, block_nx/4: one z-chunk of
 * that many planes per CTA (3-D only) — keeps the fastest pair for this
 * context and returns the z-chunk (amrvac_gpu_stage_variant reports the
 * variant).  Call after the state has been uploaded. */
int amrvac_gpu_autotune(amrvac_ctx *ctx, int reps, int *best_zchunk, double *best_ms);
/* Set the work distribution directly (0, 16, 8 or 4), e.g. from a cache. */
int amrvac_gpu_set_zchunk(amrvac_ctx *ctx, int zchunk);
/* Stage-kernel variants: 0 is the scheme's default kernel; the 3-D MHD
 * HLLD + cada3 + Einfeldt + GLM scheme at block_nx 16 has three more —
 * threads per CTA, the CTAs per SM the registers are capped for, and (FP64)
 * asynchronous bulk-copy staging of the next conserved plane.  Select one
 * (e.g. from a cache), or read the current one with its parameters. */
int amrvac_gpu_set_stage_variant(amrvac_ctx *ctx, int var);
int amrvac_gpu_stage_variant(amrvac_ctx *ctx, int *var, int *nvar, int *threads, int *ctas_per_sm, int *async);
/* Read back the last step's dt, cmax_global and global_time (synchronises). */
int amrvac_gpu_get_time(amrvac_ctx *ctx, double *dt, double *cmax_global, double *global_time);

/* Status word (OR of AMRVAC_ST_*), sticky.  Synchronises. */
int amrvac_gpu_status(amrvac_ctx *ctx, uint32_t *flags);
int amrvac_gpu_clear_status(amrvac_ctx *ctx);
int amrvac_gpu_synchronize(amrvac_ctx *ctx);
/* The context's cudaStream_t (as void*), for event timing by the caller. */
int amrvac_gpu_stream(amrvac_ctx *ctx, void **stream);
/* Device pointer of register reg (layout pool[block][var][z][y][x], 16^ndim). */
int amrvac_gpu_register_ptr(amrvac_ctx *ctx, int reg, double **dptr);
/* Number of kernel launches issued by this context since creation. */
int64_t amrvac_gpu_launch_count(const amrvac_ctx *ctx);
/* Text of the last error on this thread (empty if none). */
const char *amrvac_gpu_last_error(void);

/* Per-routine entry points over n independent faces / states (host arrays,
 * state-major [n][nw]); used to test phys_get_flux (mhd 3810-3889 / hd
 * 1097-1146), phys_get_cbounds (mhd 3037-3127 / hd 891-1001) and the
 * Riemann solvers (src/mod_finite_volume.t:348-729) one routine at a time.
 * idim is 1-based as in the reference. */
int amrvac_gpu_get_flux_points(amrvac_ctx *ctx, int n, const double *wc, const double *wp, int idim,
                               double cmax_global, double *f);
int amrvac_gpu_get_cbounds_points(amrvac_ctx *ctx, int n, const double *wlc, const double *wrc,
                                  const double *wlp, const double *wrp, int idim, double *cmax,
                                  double *cmin);
int amrvac_gpu_riemann_points(amrvac_ctx *ctx, int n, const double *wlp, const double *wrp, int idim,
                              double cmax_global, double *f);
/* The FP64 reciprocal and quotient every stage kernel uses in place of the
 * reference's divisions, on n host points: q = x/y, r = 1/y (Newton-Raphson
 * from the hardware seed, with IEEE division outside its range), and the
 * seed itself.  No counterpart in the reference (its divisions are IEEE);
 * used to test the device arithmetic against IEEE division. */
int amrvac_gpu_div_points(int n, const double *x, const double *y, double *q, double *r, double *seed);

/* CFL reduction without any device allocation (no counterpart in the
 * reference).  For callers that must not call cudaMalloc/cudaFree: host codes
 * whose device memory is owned by another runtime (OpenACC / CUDA Fortran
 * data regions, a framework's caching allocator) and so cannot create an
 * amrvac_ctx.  Computes what amrvac_gpu_getdt computes — dt from courantpar
 * and cmax_global — over nblocks blocks that the caller holds on the current
 * device in the register layout w_dev[block][var][z][y][x] (block_nx^ndim
 * cells, interior only; block_nx even, >= 4, the same in every direction),
 * with dx the host array [nblocks][3].  Uses only
 * cfg->physics, ndim, ndir, block_nx, gamma, typedivbfix, courantpar,
 * type_courant and dtmin.  Runs on `stream` (a cudaStream_t; NULL = the
 * default stream) and synchronises it.
 * Scratch: a fixed device array inside the library (1.25 MiB per GPU, held
 * until exit); nblocks above AMRVAC_NOALLOC_MAX_BLOCKS is refused with
 * AMRVAC_E_ARG.  The first call on a device looks up that array's address, so
 * make it before any stream capture; the library keeps that address for the
 * life of the process, so a cudaDeviceReset on that device invalidates it (do
 * not call this entry point after one).  All calls share the array: calls that
 * overlap on the GPU race.  Returns AMRVAC_ST_DT_TOO_SMALL if dt < dtmin. */
#define AMRVAC_NOALLOC_MAX_BLOCKS 32768
int amrvac_gpu_getdt_noalloc(const amrvac_cfg *cfg, const double *w_dev, int nblocks, const double *dx,
                             void *stream, double *dt, double *cmax_global);

/* ---- AMR decisions --------------------------------------------------------
 * Löhner error estimator (lohner_grid, src/amr/mod_errest.t:63-200,
 * refine_criterion 3) on register reg, all blocks: flags[b] = 1 if the block
 * should refine (some cell has error >= refine_threshold(level) and level <
 * refine_max_level), 2 if it may coarsen (every cell has error <=
 * derefine_ratio(level) * refine_threshold(level) and level > 1).  weight and
 * logflag: w_refine_weight and logflag per conserved variable ([nw]; logflag
 * may be NULL); refine_threshold, derefine_ratio, amr_wavefilter: per level
 * ([refine_max_level]); block_level: 1-based level per block (NULL = all 1);
 * errmax (may be NULL): the largest error of each block.  Host arrays;
 * synchronous.  Ghost values are those of getbc (same-level neighbours and
 * physical boundaries). */
int amrvac_gpu_lohner(amrvac_ctx *ctx, int reg, const double *weight, const int *logflag, int refine_max_level,
                      const double *refine_threshold, const double *derefine_ratio, const double *amr_wavefilter,
                      const int *block_level, int *flags, double *errmax);

/* ---- Discrete adjoint (no counterpart in the reference) -------------------
 * One step with a given dt (the configured RK stages, no setdt): the forward
 * map of the adjoint, whose dt sequence is frozen. */
int amrvac_gpu_step_dt(amrvac_ctx *ctx, double dt);
/* Copy a whole register to (to_register = 0) or from (1) the caller's device
 * buffer dev (register layout [block][var][y][x], 16^ndim per block). */
int amrvac_gpu_register_copy(amrvac_ctx *ctx, int reg, double *dev, int to_register);
/* One step with a given dt whose stage inputs and result are the caller's
 * device buffers (register layout), so that a checkpointed sweep keeps every
 * stage input without copies: the stages of amrvac_gpu_step_dt read u0 = U^n
 * and write u1, u2 (the inputs of stages 2 and 3; u2 unused for twostep) and
 * unew = U^{n+1}, which may be u0; unew NULL skips the last stage.  threestep
 * or twostep ssprk2, single-level unsplit grids; the registers are not
 * touched.  Asynchronous on the context stream. */
int amrvac_gpu_step_dt_states(amrvac_ctx *ctx, double dt, const double *u0, double *u1, double *u2, double *unew);
/* Adjoint of one step U^n -> U^{n+1} at frozen dt, with U^n in register 0:
 * lam (device, register layout) holds dL/dU^{n+1} on entry and dL/dU^n on
 * return; gamma_part (device, [nblocks]) accumulates dL/dgamma of the step
 * per block (sum it for the total).  Recomputes the stage inputs in
 * registers 1 and 2.  2-D hydrodynamics, HLL or HLLC with minmod or vanleer,
 * Einfeldt bounds, FP64, periodic or cont boundaries, uniform dx, threestep
 * or twostep.  Asynchronous on the context stream. */
int amrvac_gpu_adjoint_step(amrvac_ctx *ctx, double *lam, double dt, double *gamma_part);
/* The same with the step's stage inputs supplied by the caller (device,
 * register layout): u0 = U^n, u1 and u2 the inputs of stages 2 and 3 (the
 * contents of registers 1 and 2 after amrvac_gpu_step_dt from U^n; u2 unused
 * for twostep).  No stage is recomputed and the registers are not touched. */
int amrvac_gpu_adjoint_step_states(amrvac_ctx *ctx, const double *u0, const double *u1, const double *u2,
                                   double *lam, double dt, double *gamma_part);

/* ---- Batched ensembles (no counterpart in the reference) ------------------
 * Many independent hydrodynamics runs advanced together: 1-D and 2-D
 * instances of uneven sizes, each a uniform level-1 grid of 16^d blocks with
 * its own Riemann solver, limiter, end time and CFL time step, all advanced by
 * one persistent kernel launch per RK stage.  Each instance follows the
 * reference's time loop (src/amrvac.t:241-343): setdt (maxsum, dtmin check,
 * final_dt_reduction, src/mod_dt.t:10-99), exit when time_max is reached,
 * advance.  Shared by all instances (from amrvac_cfg): gamma, typeboundspeed,
 * courantpar, cada3_radius, tvdlfeps, small values, time_stepper,
 * ssprk_order, dtmin, typeboundary (periodic or cont per side) and
 * precision.  Block arrays are the reference's w(ixG^S,1:nw) per block with
 * nw = ndim + 2 (rho, m(1:ndim), e), blocks x-fastest within an instance. */
typedef struct amrvac_ens amrvac_ens;
typedef struct amrvac_ens_instance {
  int ndim;              /* 1 or 2 */
  int domain_nx[2];      /* cells per direction, multiples of 16 */
  double xprobmin[2], xprobmax[2];
  int flux_scheme;       /* AMRVAC_FS_TVDLF, _HLL or _HLLC */
  int limiter;           /* AMRVAC_LIM_* */
  double time_max;
} amrvac_ens_instance;
int amrvac_ens_create(const amrvac_cfg *cfg, int ninst, const amrvac_ens_instance *inst, amrvac_ens **out);
int amrvac_ens_destroy(amrvac_ens *ens);
/* Number of blocks of instance i. */
int amrvac_ens_nblocks(const amrvac_ens *ens, int inst);
/* Instance state in / out (ghosted block arrays; ghosts are ignored on upload
 * and filled as getbc would on download).  Synchronous. */
int amrvac_ens_upload(amrvac_ens *ens, int inst, const double *w);
int amrvac_ens_download(amrvac_ens *ens, int inst, double *w);
/* time = 0, steps = 0, all instances active. */
int amrvac_ens_reset_time(amrvac_ens *ens);
/* One step of every active instance (asynchronous). */
int amrvac_ens_step(amrvac_ens *ens);
/* Steps in CUDA-graph chunks of `chunk` steps until every instance has
 * reached its time_max or max_steps steps were issued; finished instances are
 * dropped from the work list between chunks.  Returns the steps issued and the
 * number of instances still running. */
int amrvac_ens_run(amrvac_ens *ens, int max_steps, int chunk, int *steps_taken, int *nactive);
/* Per-instance time, last dt, steps taken, done flag (arrays of ninst; any may
 * be NULL).  Synchronises. */
int amrvac_ens_state(amrvac_ens *ens, double *t, double *dt, int *steps, int *done);
/* Sticky status (OR of AMRVAC_ST_*) and per-instance status (may be NULL). */
int amrvac_ens_status(amrvac_ens *ens, uint32_t *flags, uint32_t *inst_flags);
/* CTAs of each stage launch (0 = one resident wave), and the current value. */
int amrvac_ens_set_grid(amrvac_ens *ens, int ctas);
int amrvac_ens_grid(const amrvac_ens *ens, int *ctas, int *wave);
/* Stage-kernel variant 0, 1 or 2, each one CTA per SM denser than the last
 * (FP64: two CTAs per SM at 96 registers, three at 72 or four at 56; mixed:
 * three at 72, four at 56 or five at 40).  Same arithmetic, bit-identical
 * results. */
int amrvac_ens_set_variant(amrvac_ens *ens, int var);
int amrvac_ens_variant(const amrvac_ens *ens, int *var, int *nvar, int *ctas_per_sm);
/* Times one stage for every variant and candidate grid size on the current
 * state (left unchanged) and keeps the fastest pair. */
int amrvac_ens_autotune(amrvac_ens *ens, int reps, int *best_ctas, double *best_ms);
int amrvac_ens_stream(amrvac_ens *ens, void **stream);
int64_t amrvac_ens_launch_count(const amrvac_ens *ens);

/* Same-resolution ghost-fill index maps ixS_srl_ / ixR_srl_ of init_bc
 * (src/mod_ghostcells_update.t:150-162), 0-based inclusive, for i=-1,0,1
 * at index i+1. */
int amrvac_gpu_srl_maps(int nghost, int block_nx, int *s_min, int *s_max, int *r_min, int *r_max);

#ifdef __cplusplus
}
#endif
#endif /* AMRVAC_GPU_H */
