/*
 * CPU oracle for the MPI-AMRVAC per-block finite-volume update.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is a plain FP64 restatement of the
 * reference Fortran routines (cited per function in amrvac_oracle.cpp).  It is
 * the checker that the CUDA path is compared against; it is never linked into,
 * loaded by, or called from the product library (libamrvac_gpu.so).  Only the
 * tests, the smoke check and the CPU-baseline leg of bench.py load it.
 *
 * Array convention: every block array is the Fortran array w(ixG^S,1:nw) in
 * column-major order (x fastest, variable slowest), 0-based, ghost cells
 * included.  Unused dimensions (ndim < 3) have extent 1.
 */
#ifndef AMRVAC_ORACLE_H
#define AMRVAC_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Flux scheme ids: values of the reference's fs_* parameters are not used;
 * these are this oracle's own (the names follow mod_finite_volume.t). */
enum { ORC_FS_TVDLF = 1, ORC_FS_HLL = 2, ORC_FS_HLLC = 3, ORC_FS_HLLD = 4, ORC_FS_TVDMU = 5 };
/* Limiter ids follow src/limiter/mod_limiter.t:14-24. */
enum { ORC_LIM_MINMOD = 1, ORC_LIM_WOODWARD = 2, ORC_LIM_MCBETA = 3,
       ORC_LIM_SUPERBEE = 4, ORC_LIM_VANLEER = 5, ORC_LIM_ALBADA = 6,
       ORC_LIM_KOREN = 7, ORC_LIM_CADA = 8, ORC_LIM_CADA3 = 9, ORC_LIM_SCHMID = 10, ORC_LIM_VENK = 11, ORC_LIM_MP5 = 13,
       ORC_LIM_WENO3 = 14, ORC_LIM_WENOYC3 = 15,
       ORC_LIM_WENO5 = 16, ORC_LIM_WENOZ5 = 18, ORC_LIM_WENOZP5 = 20 };
/* boundspeed ids follow src/io/mod_input_output.t:1632-1641. */
enum { ORC_BS_EINFELDT = 1, ORC_BS_CMAXMEAN = 2, ORC_BS_CMAXLEFTRIGHT = 3 };
/* divB ids follow src/mhd/mod_mhd_phys.t divb_* parameters. */
enum { ORC_DIVB_NONE = 0, ORC_DIVB_GLM = 1, ORC_DIVB_LINDE = 4 };
/* Courant types follow mod_global_parameters type_maxsum/summax/minimum. */
enum { ORC_COURANT_MAXSUM = 1, ORC_COURANT_SUMMAX = 2, ORC_COURANT_MINIMUM = 3 };
/* Physical boundary types (subset of mod_boundary_conditions bc_*). */
enum { ORC_BC_PERIODIC = 0, ORC_BC_CONT = 1, ORC_BC_SYMM = 2, ORC_BC_ASYMM = 3 };
/* Status bits returned by the oracle (mirror the product's runtime flags). */
enum { ORC_ST_SMALL_VALUE = 1, ORC_ST_DT_TOO_SMALL = 4 };

typedef struct {
  int ndim, ndir;
  int physics;            /* 0 = hd, 1 = mhd */
  int nw;                 /* number of flux variables (nwflux) */
  int nghost;
  int block_nx[3];
  double gamma;
  int flux_scheme;
  int limiter;
  int boundspeed;
  int divb;               /* mhd only */
  double glm_alpha;
  int glm_extended;
  double courantpar;
  int type_courant;
  double cada3_radius;
  double tvdlfeps;
  int fix_small_values;
  int check_small_values;
  int small_values_method;/* 0 = error, 1 = replace, 2 = average */
  double small_density, small_pressure;
  double divbdiff;
  int ssprk_order;        /* 3 (Gottlieb-Shu) or 2 */
  int time_stepper;       /* 2 twostep, 3 threestep (0 means 3), 4 fourstep */
  int time_integrator;    /* twostep: 0 Predictor_Corrector, 2 ssprk2; fourstep: 0 ssprk4, 1 rk4 */
  int dimsplit;           /* 0 unsplit, 1 'xyyx', 2 'xy' */
  double schmid_rad[3];   /* schmid2 limiter radii per direction */
  int schmid_global;      /* schmid1: a2max_global from every getdt instead */
  int small_values_daverage; /* cube half-width of the 'average' fix (0 means 1) */
} orc_cfg;

/* Number of flux variables implied by cfg (sets cfg->nw too). */
int orc_cfg_finalize(orc_cfg *cfg);

/* --- per-block routines (one block, Fortran layout, ghost cells included) --- */

/* finite_volume (src/mod_finite_volume.t:116-339) on one block: reads wct,
 * updates wnew on the interior.  dx[ndim]; cmax_global used by GLM.
 * Returns status bits. */
int orc_finite_volume(const orc_cfg *cfg, const double *wct, double *wnew,
                      double qdt, double dtfactor, const double *dx,
                      double cmax_global);

/* getdt_courant (src/mod_dt.t:160-287) on one block: returns dtnew and
 * updates *cmax_max (running max of cmax over the interior). */
int orc_getdt_block(const orc_cfg *cfg, const double *w, const double *dx,
                    double *dtnew, double *cmax_max);

/* Primitive <-> conserved conversion over the whole block array. */
void orc_to_primitive(const orc_cfg *cfg, double *w);
void orc_to_conserved(const orc_cfg *cfg, double *w);

/* Pointwise physics for per-routine parity tests.  Arrays of n states, each
 * state nw values contiguous (state-major).  idim is 1-based. */
void orc_get_flux_points(const orc_cfg *cfg, int n, const double *wc,
                         const double *wp, int idim, double cmax_global,
                         double *f);
void orc_get_cbounds_points(const orc_cfg *cfg, int n, const double *wlc,
                            const double *wrc, const double *wlp,
                            const double *wrp, int idim, double *cmax,
                            double *cmin);
/* Riemann flux at n faces from L/R primitive states (applies to_conserved,
 * modify_wLR, flux, cbounds and the configured solver). */
void orc_riemann_points(const orc_cfg *cfg, int n, const double *wlp_in,
                        const double *wrp_in, int idim, double cmax_global,
                        double *f);
/* dwlimiter2 on a 1-D line of n centred differences; ldw/rdw defined on
 * indices 1..n-1 (index 0 untouched). */
void orc_limiter_line(const orc_cfg *cfg, int n, const double *dwc,
                      double dxlevel, double *ldw, double *rdw);

/* --- uniform-grid driver (level 1 only, no AMR) --- */
typedef struct orc_grid orc_grid;

/* bc[2*ndim]: min1,max1,min2,max2,...  Block order: x fastest. */
orc_grid *orc_grid_create(const orc_cfg *cfg, const int *domain_nx,
                          const double *xprobmin, const double *xprobmax,
                          const int *bc);
void orc_grid_destroy(orc_grid *g);
int orc_grid_nblocks(const orc_grid *g);
/* Block geometry: block index -> (ig1,ig2,ig3) 0-based, and cell size. */
void orc_grid_block_index(const orc_grid *g, int ib, int *ig);
void orc_grid_dx(const orc_grid *g, double *dx);
/* Cell-centre coordinate x(i, idim) for local 0-based index i of block ib. */
double orc_grid_x(const orc_grid *g, int ib, int idim, int i);
/* Copy block arrays in/out (nw_total = cfg nw). */
void orc_grid_set_block(orc_grid *g, int ib, const double *w);
void orc_grid_get_block(const orc_grid *g, int ib, double *w);
/* getbc (src/mod_ghostcells_update.t:350-565, srl + physical BC). */
void orc_grid_getbc(orc_grid *g);
/* setdt CFL part only: dt = min over blocks; cmax_global = max cmax. */
int orc_grid_getdt(orc_grid *g, double *dt, double *cmax_global);
/* One full step with the configured stepper (SSPRK3 by default), including
 * getbc after every stage.  nthreads: OpenMP threads (<=0: default). */
int orc_grid_advance(orc_grid *g, double dt, double cmax_global, int nthreads);
/* One explicit stage: psb(ixO) = psb + fluxes(psa); reg ids 0..2 select
 * ps/ps1/ps2.  Exposed for per-stage tests. */
int orc_grid_advect1(orc_grid *g, int reg_a, int reg_b, double qdt,
                     double dtfactor, double cmax_global, int nthreads);
void orc_grid_copy_reg(orc_grid *g, int dst, int src);
void orc_grid_combine_reg(orc_grid *g, int dst, double a, int ra, double b, int rb);
/* Volume averages of w**power over the interior (printlog_regression_test). */
void orc_grid_volume_average(const orc_grid *g, int power, double *mean);

/* Index maps of the same-resolution ghost fill, 0-based inclusive bounds per
 * dimension for direction i in {-1,0,1}: ixS_srl / ixR_srl
 * (src/mod_ghostcells_update.t:150-162). out[3][2] per direction. */
void orc_srl_maps(int nghost, int block_nx, int *s_min, int *s_max,
                  int *r_min, int *r_max);

/* --- problems used by the golden-log regression tests --- */
/* Field loop 2.5D (tests/mhd/field_loop_2.5D/mod_usr.t), iprob=1.  Runs to
 * time_max writing one regression-log row every dtsave; rows[nrow_max][ncol]
 * with ncol = 1 + 2*(nw+3).  Returns number of rows, or -status on crash. */
int orc_run_field_loop(const orc_cfg *cfg, double courantpar, double time_max,
                       double dtsave, int nrow_max, double *rows, int nthreads);

/* Operation counter (+,-,*,/,sqrt,exp) of one finite_volume stage of one
 * block run in the counting scalar type; returns flops per interior cell. */
double orc_count_flops_stage(const orc_cfg *cfg, const double *wct,
                             const double *wnew, double qdt, const double *dx,
                             double cmax_global);
double orc_count_flops_getdt(const orc_cfg *cfg, const double *w,
                             const double *dx);

/* Forward-mode (dual-number) reference gradient: from the conserved block
 * arrays w0 (ghosted, nblocks x bsize) run nsteps SSP-RK3 steps with the dt
 * sequence dts (frozen), seeded with the direction (dw0, dgamma); loss = sum
 * over interior cells of mask * rho^2 (mask: nblocks x cells of a block,
 * ghosted layout).  Returns status; loss and its directional derivative in
 * *loss / *dloss; w_final (optional) the final conserved arrays. */
int orc_dual_run(const orc_cfg *cfg, const int *domain_nx, const double *xprobmin,
                 const double *xprobmax, const int *bc, const double *w0, const double *dw0,
                 double dgamma, int nsteps, const double *dts, const double *mask, int nthreads,
                 double *loss, double *dloss, double *w_final);

/* Löhner error estimator (lohner_grid, src/amr/mod_errest.t:63-200) of one
 * ghosted block: error over the interior (x fastest, optional) and the
 * reference's refine / coarsen decision for the block. */
void orc_lohner_block(const orc_cfg *cfg, const double *w, const double *weight, const int *logflag,
                      double wavefilter, double threshold, double derefine, int level, int refine_max_level,
                      double *error, int *refine, int *coarsen);

/* --- multi-level (AMR) grid: a static 2:1-balanced hierarchy of leaves --- */
typedef struct orc_amr orc_amr;
/* leaf[4*b] = level (1-based), leaf[4*b+1..3] = block index at that level
 * (0-based); nbase: level-1 blocks per direction; bc per side (one kind for
 * all variables), physical ghosts filled with current data. */
orc_amr *orc_amr_create(const orc_cfg *cfg, const int *nbase, const double *xprobmin,
                        const double *xprobmax, int nleaf, const int *leaf,
                        const int *bc /* [6] ORC_BC_* per side, NULL: periodic */);
void orc_amr_destroy(orc_amr *a);
/* ntype[b*27+q]: 0 boundary, 1 coarse, 2 sibling, 3 fine; nid: the sibling or
 * coarse block; child[(b*27+q)*8 + cbits]: fine neighbours by child position. */
int orc_amr_neighbors(const orc_amr *a, int *ntype, int *nid, int *child);
void orc_amr_set_block(orc_amr *a, int b, const double *w);
void orc_amr_get_block(const orc_amr *a, int reg, int b, double *w);
void orc_amr_getbc(orc_amr *a);
int orc_amr_getdt(orc_amr *a, double *dt, double *cmax_global);
int orc_amr_advect1(orc_amr *a, int reg_a, int reg_b, double qdt, double dtfactor, double cmax_global,
                    int nthreads);
void orc_amr_combine_reg(orc_amr *a, int dst, double ca, int ra, double cb, int rb);
int orc_amr_advance(orc_amr *a, double dt, double cmax_global, int nthreads);
/* Regrid (amr_coarsen_refine): a new grid whose register 0 comes from the old
 * grid's register 0 (after getbc) by op[9*b]: {0, old} copy, {1, old parent,
 * child bits} prolong_2nd, {2, old children in child-bit order} coarsen_grid.
 * The caller runs getbc on the new grid. */
orc_amr *orc_amr_remap(const orc_amr *old, int nleaf, const int *leaf, const int *op);

#ifdef __cplusplus
}
#endif
#endif
