// C ABI of the B200 finite-volume block update (declared in include/amrvac_gpu.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/amrvac_gpu.h"
#include "adjoint.cuh"
#include "amr.cuh"
#include "aux.cuh"
#include "kernels.cuh"

using namespace amrvac;

namespace {

thread_local std::string g_err;

int fail(int code, const std::string &msg) {
  g_err = msg;
  return code;
}

int cuda_fail(cudaError_t e, const char *where) {
  g_err = std::string(where) + ": " + cudaGetErrorString(e);
  return AMRVAC_E_CUDA;
}

#define CK(call)                                   \
  do {                                             \
    cudaError_t e_ = (call);                       \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call); \
  } while (0)

int nw_of(const amrvac_cfg *c) {
  if (c->physics == 1) {
    const bool glm = c->typedivbfix == AMRVAC_DIVB_GLM && c->ndim > 1;
    return 2 * c->ndir + 2 + (glm ? 1 : 0);
  }
  return c->ndir + 2;
}

// init_bc same-resolution maps (src/mod_ghostcells_update.t:150-162), 0-based.
void srl_maps_1d(int ng, int nx, int *smin, int *smax, int *rmin, int *rmax) {
  const int ixMmin = ng + 1, ixMmax = ng + nx, ixGmax = nx + 2 * ng;
  const int s_min[3] = {ixMmin, ixMmin, ixMmax + 1 - ng};
  const int s_max[3] = {ixMmin - 1 + ng, ixMmax, ixMmax};
  const int r_min[3] = {1, ixMmin, ixMmax + 1};
  const int r_max[3] = {ng, ixMmax, ixGmax};
  for (int q = 0; q < 3; ++q) {
    smin[q] = s_min[q] - 1; smax[q] = s_max[q] - 1;
    rmin[q] = r_min[q] - 1; rmax[q] = r_max[q] - 1;
  }
}

}  // namespace

struct amrvac_ctx {
  amrvac_cfg cfg;
  int nw = 0;
  PhysParams P;
  KernelSet ks;
  BcSpec bc;
  SrlMaps maps;
  cudaStream_t stream = nullptr;
  int nblocks = 0;
  int bn = 16;           // block edge (block_nx)
  size_t per_block = 0;  // doubles per block per variable (bn^ndim)
  double *pool[4] = {nullptr, nullptr, nullptr, nullptr};  // ps, ps1, ps2 (+ ps3 for rk4)
  int nreg = 3;                          // registers allocated
  int *d_nbr = nullptr;
  double *d_dx = nullptr;
  double *d_scal = nullptr;              // see setdt_finalize_kernel
  unsigned long long *d_red = nullptr;   // getdt reduction accumulators
  uint32_t *d_status = nullptr;
  uint32_t *d_block_status = nullptr;
  double *d_stage = nullptr;             // upload/download staging
  size_t stage_doubles = 0;
  cudaGraphExec_t graph = nullptr;
  int64_t launches = 0;
  int64_t graph_nodes = 0;
  int zchunk = 0;          // 0: persistent plane ranges; 16/8/4: one z-chunk per CTA
  int sweep = -1;          // dimensional splitting: the current sweep of the step (-1: unsplit)
  bool fixed_dir = false;  // sweep is a direction (amrvac_gpu_advect1_dim), not a sweep index
  int wave_ctas = 1;       // resident stage CTAs on the device (one wave)
  int var = 0;             // stage-kernel variant (KernelSet::stage_v; chosen by the autotuner)
  // small_values_method 'average': whole-block recomputation of the flagged
  // blocks (smallavg.cu), its scratch, and a pre-stage copy of a register
  // the stage writes in place (the output's ghost values are the RK
  // combination of the inputs' values from before the stage)
  bool sv_on = false;
  SvSet sv;
  double *sv_scratch = nullptr;
  size_t sv_per_cta = 0;
  int sv_ctas = 0;
  double *sv_snap = nullptr;
  int wave_v[KernelSet::MAXVAR] = {1, 1, 1, 1};  // one wave of each variant
  std::vector<double> h_dx;            // [nblocks][3] cell sizes (host copy)
  double *d_adj[3] = {nullptr, nullptr, nullptr};  // adjoint work registers (lazily)
  int *d_amr_int = nullptr;            // [2][nblocks] levels, flags (Löhner, lazily)
  double *d_amr_err = nullptr;         // [nblocks] largest error per block
  bool adj_prepared = false;
  bool a2max_set = false;  // schmid1: a getdt has reduced a2max_global since the last upload / grid change
  struct AmrDev *amr = nullptr;        // multi-level grid (amrvac_gpu_set_amr_grid)
  // Capacities (in blocks or elements) of the buffers that a new block set or
  // a regrid reuses while they are large enough (grown by 25 % otherwise).
  size_t pool_cap = 0, nbr_cap = 0, amr_int_cap = 0;
  double *amr_gbuf = nullptr, *amr_pflux = nullptr, *amr_bxmin = nullptr;
  int *amr_ints = nullptr;
  size_t amr_gbuf_cap = 0, amr_pflux_cap = 0, amr_bxmin_cap = 0, amr_ints_cap = 0;
};

// Grow-only device buffer: reallocates (without keeping the contents) only
// when need exceeds the capacity, then with 25 % headroom.
template <class T>
static cudaError_t ensure_capacity(T **p, size_t *cap, size_t need) {
  if (*p && need <= *cap) return cudaSuccess;
  cudaFree(*p);
  *p = nullptr;
  *cap = 0;
  const size_t n = need + need / 4 + 1;
  const cudaError_t e = cudaMalloc(p, sizeof(T) * n);
  if (e == cudaSuccess) *cap = n;
  return e;
}

// Device copy of a static multi-level grid: neighbour kinds, per-level owner
// maps, ghost buffers of the blocks next to a level jump and their boundary
// face fluxes.
struct AmrDev {
  int nslots = 0;
  int *d_int = nullptr;       // iblocks, gslot, face, ntype, level, ig, child, owner
  double *d_bxmin = nullptr;  // [nblocks*3]
  double *gbuf = nullptr;     // [slot][var][(bn+4)^d]
  double *pflux = nullptr;    // [slot][2*ndim][var][bn*bn]
  AmrGhostArgs G;
  AmrFixArgs F;
  int *d_face = nullptr, *d_gslot = nullptr;
  std::vector<int> h_leaf;    // [nblocks][4] level, ig0, ig1, ig2 (regrid checks)
  int nbase[3] = {1, 1, 1};
  double xmin[3] = {0, 0, 0}, xmax[3] = {1, 1, 1};
  // the device buffers belong to the context (amr_* fields), reused across regrids
};

namespace {

// twostep Predictor_Corrector predicts with the MUSCL-Hancock scheme when the
// flux scheme is tvdlf (typepred1 = fs_hancock, src/io/mod_input_output.t:
// 787-797); the other schemes predict with their own finite_volume.
bool uses_hancock(const amrvac_cfg &k) {
  return k.time_stepper == AMRVAC_TS_TWOSTEP && k.time_integrator == AMRVAC_TI_DEFAULT &&
         (k.flux_scheme == AMRVAC_FS_TVDLF || k.flux_scheme == AMRVAC_FS_TVDMU);
}

int check_ctx(amrvac_ctx *c, bool need_blocks) {
  if (!c) return fail(AMRVAC_E_ARG, "null context");
  if (need_blocks && c->nblocks == 0) return fail(AMRVAC_E_STATE, "no blocks set (amrvac_gpu_set_blocks)");
  return 0;
}

StageArgs stage_args(amrvac_ctx *c, int reg_ct, int reg_new, int reg_base, double a, double b,
                     double dtfactor) {
  StageArgs A;
  std::memset(&A, 0, sizeof(A));
  A.uin = c->pool[reg_ct];
  A.ubase = c->pool[reg_base];
  A.uout = c->pool[reg_new];
  A.a_base = a;
  A.b_in = b;
  A.dtfactor = dtfactor;
  A.dt_dev = c->d_scal + 0;
  A.cmax_dev = c->d_scal + 1;
  A.nbr = c->d_nbr;
  A.dxb = c->d_dx;
  A.nblocks = c->nblocks;
  A.zchunk = c->zchunk;
  for (int s = 0; s < 6; ++s) {
    A.bc_kind[s] = c->bc.kind[s];
    A.bc_flip[s] = c->bc.flip[s];
  }
  A.status = c->d_status;
  A.block_status = c->d_block_status;
  A.P = c->P;
  A.sweep = c->sweep;
  A.split_xy = c->fixed_dir || c->cfg.dimsplit == 2;
  A.bn = c->bn;
  if (c->amr) {
    A.gbuf = c->amr->gbuf;
    A.pflux = c->amr->pflux;
    A.gslot = c->amr->d_gslot;
    A.amr_face = c->amr->d_face;
  }
  return A;
}

// Ghost values of the level-jump directions of register reg (restriction and
// prolongation) into the ghost buffers.
int launch_amr_ghost_pass(amrvac_ctx *c, int reg) {
  AmrGhostArgs G = c->amr->G;
  G.u = c->pool[reg];
  CK(launch_amr_ghosts(G, c->amr->nslots, c->cfg.ndim, c->stream));
  ++c->launches;
  return 0;
}

// fix: apply fix_conserve after the stage on a multi-level grid (the
// reference's predictor step skips it: fix_conserve_at_step = .false.).
// hancock: the MUSCL-Hancock predictor instead of finite_volume (no flux fix,
// no block restore on a small-value crash).
int launch_stage(amrvac_ctx *c, int reg_ct, int reg_new, int reg_base, double a, double b, double dtfactor,
                 bool fix = true, bool hancock = false) {
  if (hancock && !c->ks.hancock) return fail(AMRVAC_E_UNSUPPORTED, "no Hancock predictor for this configuration");
  if (c->amr)
    if (int r = launch_amr_ghost_pass(c, reg_ct)) return r;
  StageArgs A = stage_args(c, reg_ct, reg_new, reg_base, a, b, dtfactor);
  // tile-planes: tiles per block plane x z-planes (3-D)
  const int bn = c->bn, ntile = (bn / tile_edge(bn)) * (bn / tile_edge(bn));
  const long planes = (long)c->nblocks * ntile * (c->cfg.ndim == 3 ? bn : 1);
  int nctas;
  if (c->zchunk > 0) nctas = c->nblocks * ntile * (c->cfg.ndim == 3 ? bn / c->zchunk : 1);
  else nctas = (int)std::min<long>(planes, hancock ? c->wave_ctas : c->wave_v[c->var]);
  const bool restore = !hancock && c->P.fix_small_values && c->P.small_values_method == 0;
  if (restore || c->sv_on) CK(cudaMemsetAsync(c->d_block_status, 0, sizeof(uint32_t) * c->nblocks, c->stream));
  // 'average': a register the stage overwrites in place is copied first (the
  // whole-block path reads its neighbours' values from before the stage)
  const double *snap_base = nullptr, *snap_in = nullptr;
  if (c->sv_on) {
    const size_t bytes = sizeof(double) * c->per_block * c->nw * c->nblocks;
    if (a != 0.0 && reg_base == reg_new) {
      CK(cudaMemcpyAsync(c->sv_snap, c->pool[reg_base], bytes, cudaMemcpyDeviceToDevice, c->stream));
      snap_base = c->sv_snap;
    } else if (reg_ct == reg_new) {
      CK(cudaMemcpyAsync(c->sv_snap, c->pool[reg_ct], bytes, cudaMemcpyDeviceToDevice, c->stream));
      snap_in = c->sv_snap;
    }
    CK(c->sv.detect(A, c->pool[reg_ct], c->stream));
    ++c->launches;
  }
  CK(hancock ? c->ks.hancock(A, nctas, c->stream) : c->ks.stage_v[c->var](A, nctas, c->stream));
  ++c->launches;
  if (c->sv_on) {
    CK(c->sv.stage(A, snap_base, snap_in, SvScratch{c->sv_scratch, c->sv_per_cta}, c->sv_ctas, c->stream));
    ++c->launches;
  }
  if (c->cfg.ndim == 3 && c->cfg.physics == 1 && c->cfg.typedivbfix == AMRVAC_DIVB_LINDE) {
    if (!c->ks.linde3d) return fail(AMRVAC_E_UNSUPPORTED, "no 3-D Linde kernel for this configuration");
    CK(c->ks.linde3d(A, c->stream));  // addsource2 of finite_volume / hancock
    ++c->launches;
  }
  if (hancock) return 0;
  if (restore) {
    CK(launch_restore_blocks(c->pool[reg_ct], c->pool[reg_new], c->d_block_status, c->nblocks,
                             c->per_block * c->nw, c->stream));
    ++c->launches;
  }
  if (c->amr && fix) {  // fix_conserve on the stage's output
    AmrFixArgs F = c->amr->F;
    F.w = c->pool[reg_new];
    F.sweep = c->sweep;
    F.split_xy = c->fixed_dir || c->cfg.dimsplit == 2;
    CK(launch_amr_fix(F, c->amr->nslots, c->cfg.ndim, c->stream));
    ++c->launches;
  }
  return 0;
}

// Work distribution of the 3-D stage kernel: 0 (persistent plane ranges) or
// z-chunks of zchunk planes, zchunk >= 2 dividing the block edge.
static bool valid_zchunk(int bn, int zchunk) { return zchunk == 0 || (zchunk >= 2 && bn % zchunk == 0); }

int launch_getdt(amrvac_ctx *c, int reg) {
  GetdtArgs G;
  G.u = c->pool[reg];
  G.dxb = c->d_dx;
  G.nblocks = c->nblocks;
  G.bn = c->bn;
  G.type_courant = c->cfg.type_courant;
  G.red = c->d_red;
  G.P = c->P;
  G.status = c->d_status;
  G.skip = nullptr;
  StageArgs SA;
  if (c->sv_on) {  // 'average': the blocks with a small value go through sv_getdt
    SA = stage_args(c, reg, reg, reg, 0.0, 1.0, 1.0);
    CK(cudaMemsetAsync(c->d_block_status, 0, sizeof(uint32_t) * c->nblocks, c->stream));
    CK(c->sv.detect(SA, c->pool[reg], c->stream));
    ++c->launches;
    G.skip = c->d_block_status;
  }
  CK(c->ks.getdt(G, c->stream));
  ++c->launches;
  if (c->sv_on) {
    CK(c->sv.getdt(SA, c->pool[reg], c->cfg.type_courant, c->d_red, SvScratch{c->sv_scratch, c->sv_per_cta},
                   c->sv_ctas, c->stream));
    ++c->launches;
  }
  if (c->cfg.schmid_global) {  // a2max_global for schmid1 (getdt_courant + MPI_ALLREDUCE max)
    if (c->amr)
      if (int r = launch_amr_ghost_pass(c, reg)) return r;
    CK(cudaMemsetAsync(c->d_scal + 10, 0, 3 * sizeof(double), c->stream));
    StageArgs A = stage_args(c, reg, reg, reg, 0.0, 1.0, 1.0);
    CK(c->ks.a2max(A, c->d_scal + 10, c->stream));
    ++c->launches;
    c->a2max_set = true;
  }
  return 0;
}

// schmid1 reads a2max_global, which only the getdt phase reduces: a stage
// called without a getdt on the current state would use a stale or zero
// value, so it is refused.
static int check_a2max(const amrvac_ctx *c) {
  if (c->cfg.schmid_global && !c->a2max_set)
    return fail(AMRVAC_E_STATE, "schmid1 (schmid_global): call amrvac_gpu_getdt on this state before a stage");
  return 0;
}

// fourstep (src/mod_advance.t:454-512), coefficients src/io/mod_input_output.t:
// 1036-1067.  ssprk4 in registers 0..2: ps1 = ps + b11 dt L(ps); ps2 = a21 ps
// + a22 ps1 + b22 dt L(ps1); ps1 = a31 ps + a33 ps2 + b33 dt L(ps2); ps = a41
// ps + a44 ps1 + b44 dt L(ps1).  rk4 with register 3: ps1 = ps + dt/2 L(ps),
// ps2 = ps + dt/2 L(ps1), ps3 = ps + dt L(ps2), ps = (1/3)(-ps + ps1 + 2 ps2 +
// ps3), ps = ps + dt/6 L(ps3).  ev (optional) receives an event after every
// stage.
int launch_fourstep(amrvac_ctx *c, cudaEvent_t *ev) {
  const amrvac_cfg &k = c->cfg;
  int r = 0;
  auto mark = [&](int i) { if (ev) cudaEventRecord(ev[i], c->stream); };
  if (k.time_integrator == AMRVAC_TI_RK4) {
    if ((r = launch_stage(c, 0, 1, 0, 0.0, 1.0, 0.5))) return r;
    mark(0);
    if ((r = launch_stage(c, 1, 2, 0, 1.0, 0.0, 0.5))) return r;
    mark(1);
    if ((r = launch_stage(c, 2, 3, 0, 1.0, 0.0, 1.0))) return r;
    CK(launch_rk4_combine(c->pool[0], c->pool[1], c->pool[2], c->pool[3], c->per_block * c->nw * c->nblocks,
                          c->stream));
    ++c->launches;
    mark(2);
    r = launch_stage(c, 3, 0, 0, 1.0, 0.0, 1.0 / 6.0);
    mark(3);
    return r;
  }
  double b11, b22, b33, b44, a21, a31, a41;
  if (k.ssprk_order == 2) {
    b11 = 1.0 / 3.0; b22 = 1.0 / 3.0; b33 = 1.0 / 3.0; b44 = 1.0 / 4.0; a21 = 0.0; a31 = 0.0; a41 = 1.0 / 4.0;
  } else {
    b11 = 1.0 / 2.0; b22 = 1.0 / 2.0; b33 = 1.0 / 6.0; b44 = 1.0 / 2.0; a21 = 0.0; a31 = 2.0 / 3.0; a41 = 0.0;
  }
  if ((r = launch_stage(c, 0, 1, 0, 0.0, 1.0, b11))) return r;
  mark(0);
  if ((r = launch_stage(c, 1, 2, 0, a21, 1.0 - a21, b22))) return r;
  mark(1);
  if ((r = launch_stage(c, 2, 1, 0, a31, 1.0 - a31, b33))) return r;
  mark(2);
  r = launch_stage(c, 1, 0, 0, a41, 1.0 - a41, b44);
  mark(3);
  return r;
}

// fivestep ssprk5 (src/mod_advance.t:513-557), coefficients
// src/io/mod_input_output.t:1079-1140 (ssprk_order 3: Gottlieb 2005; 2:
// Spiteri-Ruuth), on registers 0..3:
//   ps1 = ps + b11 dt L(ps)
//   ps2 = a21 ps + a22 ps1 + b22 dt L(ps1)
//   ps1 = a31 ps + a33 ps2 + b33 dt L(ps2)
//   ps3 = a53 ps2 + a54 ps1;  ps2 = a41 ps + a44 ps1 + b44 dt L(ps1)
//   ps = ps3 + a55 ps2 + (b54/b44)(ps2 - (a41 ps + a44 ps1));  ps += b55 dt L(ps2)
struct Ssprk5 {
  double b11, b22, b33, b44, b54, b55, a21, a31, a41, a53, a54, a22, a33, a44, a55;
};
Ssprk5 ssprk5_coefficients(int order) {
  Ssprk5 k;
  if (order == 2) {
    k.b11 = 0.39175222700392; k.b22 = 0.36841059262959; k.b33 = 0.25189177424738; k.b44 = 0.54497475021237;
    k.a21 = 0.44437049406734; k.a31 = 0.62010185138540; k.a41 = 0.17807995410773; k.a53 = 0.51723167208978;
    k.a22 = 1.0 - k.a21; k.a33 = 1.0 - k.a31; k.a44 = 1.0 - k.a41;
    const double rka51 = 0.00683325884039, rka54 = 0.12759831133288, rkb54 = 0.08460416338212;
    k.b54 = rkb54 - k.b44 * rka51 / k.a41;
    k.a54 = rka54 - k.a44 * rka51 / k.a41;
    k.a55 = 1.0 - k.a53 - k.a54;
    const double c2 = k.b11, c3 = k.a22 * c2 + k.b22, c4 = k.a33 * c3 + k.b33, c5 = k.a44 * c4 + k.b44;
    k.b55 = 1.0 - k.b54 - k.a53 * c3 - k.a54 * c4 - k.a55 * c5;
  } else {
    k.b11 = 0.391752226571890; k.b22 = 0.368410593050371; k.b33 = 0.251891774271694;
    k.b44 = 0.544974750228521; k.b54 = 0.063692468666290; k.b55 = 0.226007483236906;
    k.a21 = 0.444370493651235; k.a31 = 0.620101851488403; k.a41 = 0.178079954393132;
    k.a53 = 0.517231671970585; k.a54 = 0.096059710526147;
    k.a22 = 1.0 - k.a21; k.a33 = 1.0 - k.a31; k.a44 = 1.0 - k.a41; k.a55 = 1.0 - k.a53 - k.a54;
  }
  return k;
}

int launch_fivestep(amrvac_ctx *c, cudaEvent_t *ev) {
  const Ssprk5 K = ssprk5_coefficients(c->cfg.ssprk_order);
  const size_t n = c->per_block * c->nw * c->nblocks;
  int r = 0;
  auto mark = [&](int i) { if (ev) cudaEventRecord(ev[i], c->stream); };
  if ((r = launch_stage(c, 0, 1, 0, 0.0, 1.0, K.b11))) return r;
  mark(0);
  if ((r = launch_stage(c, 1, 2, 0, K.a21, K.a22, K.b22))) return r;
  mark(1);
  if ((r = launch_stage(c, 2, 1, 0, K.a31, K.a33, K.b33))) return r;
  mark(2);
  CK(launch_ssprk5_ps3(c->pool[3], c->pool[2], c->pool[1], K.a53, K.a54, n, c->stream));
  ++c->launches;
  if ((r = launch_stage(c, 1, 2, 0, K.a41, K.a44, K.b44))) return r;
  CK(launch_ssprk5_final(c->pool[0], c->pool[1], c->pool[2], c->pool[3], K.a55, K.b54 / K.b44, K.a41, K.a44, n,
                         c->stream));
  ++c->launches;
  mark(3);
  r = launch_stage(c, 2, 0, 0, 1.0, 0.0, K.b55);
  mark(4);
  return r;
}

// The configured RK stages (src/mod_advance.t:56-567) on registers 0..2.
int launch_rk(amrvac_ctx *c) {
  const amrvac_cfg &k = c->cfg;
  int r = 0;
  if (k.time_stepper == AMRVAC_TS_ONESTEP) {
    CK(cudaMemcpyAsync(c->pool[1], c->pool[0], sizeof(double) * c->per_block * c->nw * c->nblocks,
                       cudaMemcpyDeviceToDevice, c->stream));
    r = launch_stage(c, 1, 0, 0, 0.0, 1.0, 1.0);
  } else if (k.time_stepper == AMRVAC_TS_TWOSTEP) {
    if (k.time_integrator == AMRVAC_TI_SSPRK2) {
      if ((r = launch_stage(c, 0, 1, 0, 0.0, 1.0, 1.0))) return r;
      r = launch_stage(c, 1, 0, 0, 0.5, 0.5, 0.5);
    } else {  // Predictor_Corrector (src/mod_advance.t:104-111), typepred1
      if ((r = launch_stage(c, 0, 1, 0, 0.0, 1.0, 0.5, false, uses_hancock(k)))) return r;
      r = launch_stage(c, 1, 0, 0, 1.0, 0.0, 1.0);
    }
  } else if (k.time_stepper == AMRVAC_TS_FOURSTEP) {
    r = launch_fourstep(c, nullptr);
  } else if (k.time_stepper == AMRVAC_TS_FIVESTEP) {
    r = launch_fivestep(c, nullptr);
  } else {
    double b11, b22, b33, a21, a31;
    if (k.ssprk_order == 2) { b11 = 0.5; b22 = 0.5; b33 = 1.0 / 3.0; a21 = 0.0; a31 = 1.0 / 3.0; }
    else { b11 = 1.0; b22 = 1.0 / 4.0; b33 = 2.0 / 3.0; a21 = 3.0 / 4.0; a31 = 1.0 / 3.0; }
    const double a22 = 1.0 - a21, a33 = 1.0 - a31;
    if ((r = launch_stage(c, 0, 1, 0, 0.0, 1.0, b11))) return r;
    if ((r = launch_stage(c, 1, 2, 0, a21, a22, b22))) return r;
    r = launch_stage(c, 2, 0, 0, a31, a33, b33);
  }
  return r;
}

int launch_step(amrvac_ctx *c) {
  int r;
  if ((r = launch_getdt(c, 0))) return r;
  CK(launch_setdt_finalize(c->d_red, c->d_scal, c->d_status, c->stream));
  ++c->launches;
  if (c->cfg.dimsplit) {  // one full stepper per direction (src/mod_advance.t:23-45)
    for (int s = 0; s < c->cfg.ndim && !r; ++s) {
      c->sweep = s;
      r = launch_rk(c);
    }
    c->sweep = -1;
    if (r) return r;
  } else if ((r = launch_rk(c))) {
    return r;
  }
  CK(launch_advance_time(c->d_scal, c->stream));
  ++c->launches;
  return 0;
}

}  // namespace

namespace amrvac {
// Sets this thread's last-error text for entry points defined in other units.
int record_error(int code, const std::string &msg) { return fail(code, msg); }
}  // namespace amrvac

extern "C" {

const char *amrvac_gpu_last_error(void) { return g_err.c_str(); }

void amrvac_gpu_default_cfg(amrvac_cfg *c) {
  std::memset(c, 0, sizeof(*c));
  c->ndim = 2;
  c->ndir = 2;
  c->physics = 0;
  c->block_nx[0] = c->block_nx[1] = c->block_nx[2] = 16;
  c->nghostcells = 2;
  c->gamma = 5.0 / 3.0;
  c->flux_scheme = AMRVAC_FS_TVDLF;
  c->limiter = AMRVAC_LIM_MINMOD;
  c->typeboundspeed = AMRVAC_BS_EINFELDT;
  c->typedivbfix = AMRVAC_DIVB_LINDE;
  c->mhd_glm_alpha = 0.5;
  c->mhd_glm_extended = 1;
  c->divbdiff = 0.8;
  c->courantpar = 0.8;
  c->type_courant = AMRVAC_COURANT_MAXSUM;
  c->cada3_radius = 0.1;
  c->schmid_rad[0] = c->schmid_rad[1] = c->schmid_rad[2] = 1.0;
  c->tvdlfeps = 1.0;
  c->fix_small_values = 0;
  c->check_small_values = 1;
  c->small_values_method = 0;
  c->small_values_daverage = 1;
  c->time_stepper = AMRVAC_TS_THREESTEP;
  c->ssprk_order = 3;
  c->dtmin = 1.0e-10;
  c->zchunk = 0;
  c->precision = 0;
  c->slowsteps = -1;
  c->time_integrator = AMRVAC_TI_DEFAULT;
}

int amrvac_gpu_nw(const amrvac_cfg *cfg) { return cfg ? nw_of(cfg) : AMRVAC_E_ARG; }

int amrvac_gpu_srl_maps(int nghost, int block_nx, int *s_min, int *s_max, int *r_min, int *r_max) {
  if (!s_min || !s_max || !r_min || !r_max || nghost < 1 || block_nx < nghost) return AMRVAC_E_ARG;
  srl_maps_1d(nghost, block_nx, s_min, s_max, r_min, r_max);
  return 0;
}

int amrvac_gpu_create(const amrvac_cfg *cfg, amrvac_ctx **out) {
  if (!cfg || !out) return fail(AMRVAC_E_ARG, "null argument");
  *out = nullptr;
  const amrvac_cfg &k = *cfg;
  if (k.ndim < 2 || k.ndim > 3) return fail(AMRVAC_E_UNSUPPORTED, "ndim must be 2 or 3");
  if (k.ndir < k.ndim || k.ndir > 3) return fail(AMRVAC_E_UNSUPPORTED, "ndir must be in [ndim, 3]");
  const int bn = k.block_nx[0];
  for (int d = 0; d < k.ndim; ++d)
    if (k.block_nx[d] != bn) return fail(AMRVAC_E_UNSUPPORTED, "block_nx must be the same in every direction");
  if (!block_edge_built(bn))
    return fail(AMRVAC_E_UNSUPPORTED, "block_nx must be 8, 10, 12, 16 or 32 (the block edges this library is built for)");
  if (k.nghostcells < 2) return fail(AMRVAC_E_UNSUPPORTED, "nghostcells must be >= 2");
  if (k.physics != 0 && k.physics != 1) return fail(AMRVAC_E_ARG, "physics must be 0 (hd) or 1 (mhd)");
  const bool fifth = k.limiter == AMRVAC_LIM_MP5 || k.limiter == AMRVAC_LIM_WENO5 ||
                     k.limiter == AMRVAC_LIM_WENOZ5 || k.limiter == AMRVAC_LIM_WENOZP5;
  // reconstructions outside reconstruct_LR's slope-limiter branch (their own kernels)
  const bool special = fifth || k.limiter == AMRVAC_LIM_VENK || k.limiter == AMRVAC_LIM_WENO3 ||
                       k.limiter == AMRVAC_LIM_WENOYC3;
  if ((k.limiter < 1 || k.limiter > 10) && !special) return fail(AMRVAC_E_UNSUPPORTED, "limiter not supported");
  if (special && k.precision == 1) return fail(AMRVAC_E_UNSUPPORTED, "this limiter is FP64 only");
  if (bn != 16 && special)
    return fail(AMRVAC_E_UNSUPPORTED, "block_nx other than 16: the slope limiters only");
  if (fifth && k.nghostcells < 3) return fail(AMRVAC_E_ARG, "mp5 / weno5 need nghostcells >= 3");
  if (fifth && k.precision == 1) return fail(AMRVAC_E_UNSUPPORTED, "mp5 / weno5 are FP64 only");
  if (k.typeboundspeed < 1 || k.typeboundspeed > 3) return fail(AMRVAC_E_ARG, "bad typeboundspeed");
  if (k.type_courant < 1 || k.type_courant > 3) return fail(AMRVAC_E_ARG, "bad type_courant");
  if (k.time_stepper < 1 || k.time_stepper > 5) return fail(AMRVAC_E_UNSUPPORTED, "time_stepper not supported");
  if (k.time_integrator != AMRVAC_TI_DEFAULT &&
      !(k.time_stepper == AMRVAC_TS_FOURSTEP && k.time_integrator == AMRVAC_TI_RK4) &&
      !(k.time_stepper == AMRVAC_TS_TWOSTEP && k.time_integrator == AMRVAC_TI_SSPRK2))
    return fail(AMRVAC_E_UNSUPPORTED, "time_integrator not supported for this time_stepper");
  if (uses_hancock(k) && k.precision == 1)
    return fail(AMRVAC_E_UNSUPPORTED, "the Hancock predictor (twostep with tvdlf) is FP64 only");
  if ((k.time_stepper == AMRVAC_TS_THREESTEP || k.time_stepper == AMRVAC_TS_FOURSTEP ||
       k.time_stepper == AMRVAC_TS_FIVESTEP) && k.ssprk_order != 2 && k.ssprk_order != 3)
    return fail(AMRVAC_E_ARG, "ssprk_order must be 2 or 3");
  if (k.physics == 0 && k.ndir != k.ndim) return fail(AMRVAC_E_UNSUPPORTED, "hd requires ndir == ndim");
  if (k.physics == 1) {
    if (k.typedivbfix != AMRVAC_DIVB_NONE && k.typedivbfix != AMRVAC_DIVB_GLM && k.typedivbfix != AMRVAC_DIVB_LINDE)
      return fail(AMRVAC_E_UNSUPPORTED, "typedivbfix must be none, glm or linde");
  } else if (k.flux_scheme == AMRVAC_FS_HLLD) {
    return fail(AMRVAC_E_UNSUPPORTED, "hlld needs mhd");
  }
  if (k.flux_scheme < AMRVAC_FS_TVDLF || k.flux_scheme > AMRVAC_FS_TVDMU)
    return fail(AMRVAC_E_ARG, "unknown flux_scheme");
  if (k.dimsplit < 0 || k.dimsplit > 2) return fail(AMRVAC_E_ARG, "dimsplit must be 0, 1 (xyyx) or 2 (xy)");
  // The reference's unsplit TVD-MUSCL limits every direction with the states
  // reconstructed for the last one (finite_volume's flux and update loops are
  // separate); its tests run TVD-MUSCL dimensionally split only.
  if (k.flux_scheme == AMRVAC_FS_TVDMU &&
      (!k.dimsplit || k.precision == 1 || (k.physics == 1 && k.typedivbfix == AMRVAC_DIVB_GLM)))
    return fail(AMRVAC_E_UNSUPPORTED, "tvdmu: dimsplit, FP64, no GLM");
  const int nw = nw_of(cfg);
  if (nw > AMRVAC_MAX_NW) return fail(AMRVAC_E_UNSUPPORTED, "too many variables");
  if (k.precision != 0 && k.precision != 1) return fail(AMRVAC_E_ARG, "precision must be 0 (fp64) or 1 (mixed)");
  if (k.fix_small_values && (k.small_values_method < 0 || k.small_values_method > 2))
    return fail(AMRVAC_E_UNSUPPORTED, "small_values_method: error (0), replace (1) or average (2)");
  if (k.fix_small_values && k.small_values_method == 2) {
    // the whole-block path of 'average' (smallavg.cu) covers unsplit
    // finite_volume stages with the dwlimiter2 limiters and GLM or no divB
    // source; it recomputes a flagged block in FP64 in either form (the
    // mixed form decides the face-state flags in FP64: sv_near_floor)
    if (k.dimsplit) return fail(AMRVAC_E_UNSUPPORTED, "small_values_method average: unsplit stages only");
    if (k.limiter < 1 || k.limiter > 10 || k.limiter == AMRVAC_LIM_VENK)
      return fail(AMRVAC_E_UNSUPPORTED, "small_values_method average: the dwlimiter2 limiters only");
    if (k.physics == 1 && k.ndim > 1 && k.typedivbfix == AMRVAC_DIVB_LINDE)
      return fail(AMRVAC_E_UNSUPPORTED, "small_values_method average: GLM or no divB source (not linde)");
    if (uses_hancock(k)) return fail(AMRVAC_E_UNSUPPORTED, "small_values_method average: no Hancock predictor");
    if (k.small_values_daverage < 0) return fail(AMRVAC_E_ARG, "small_values_daverage must be >= 0");
  }
  amrvac_ctx *c = new amrvac_ctx();
  c->cfg = k;
  c->nreg = ((k.time_stepper == AMRVAC_TS_FOURSTEP && k.time_integrator == AMRVAC_TI_RK4) ||
             k.time_stepper == AMRVAC_TS_FIVESTEP) ? 4 : 3;
  c->nw = nw;
  c->bn = bn;
  KernelKey key{k.physics == 1, k.ndim, k.ndir, k.physics == 1 && k.typedivbfix == AMRVAC_DIVB_GLM,
                k.flux_scheme, k.limiter, k.typeboundspeed, k.precision == 1, bn};
  if (std::getenv("AMRVAC_GENERIC_KERNELS") && !special) { key.limiter = 0; key.boundspeed = 0; }
  // one kernel per family, the variant read at run time
  if (fifth && k.limiter != AMRVAC_LIM_MP5) key.limiter = LIM_WENO5;
  if (k.limiter == AMRVAC_LIM_WENOYC3) key.limiter = LIM_WENO3;
  bool found;
  if (bn != 16) {
    key.limiter = 0;  // run-time limiter and bound speed
    key.boundspeed = 0;
    found = lookup_bn8(key, &c->ks) || lookup_bn10(key, &c->ks) || lookup_bn12(key, &c->ks) ||
            lookup_bn32(key, &c->ks);
  } else {
    found = special ? (lookup_mp5_hd(key, &c->ks) || lookup_mp5_mhd(key, &c->ks))
                    : (lookup_hd(key, &c->ks) || lookup_mhd2(key, &c->ks) || lookup_mhd3(key, &c->ks));
  }
  if (!found) {
    delete c;
    return fail(AMRVAC_E_UNSUPPORTED, key.mixed ? "no mixed-precision kernel for this scheme"
                                                : "no kernel for this physics/ndim/ndir/solver combination");
  }
  if (bn == 16 && !special) add_stage_variants(key, &c->ks);
  if (k.fix_small_values && k.small_values_method == 2) {
    if (!lookup_sv(key, &c->sv)) {
      delete c;
      return fail(AMRVAC_E_UNSUPPORTED, "small_values_method average: no whole-block kernel for this scheme");
    }
    c->sv_on = true;
  }
  cudaError_t e0;
  PhysParams &P = c->P;
  P.gamma = k.gamma;
  P.gamma_1 = k.gamma - 1.0;
  P.inv_gamma_1 = 1.0 / (k.gamma - 1.0);
  P.small_density = k.small_density;
  P.small_pressure = k.small_pressure;
  P.small_e = k.physics == 1 ? k.small_pressure * P.inv_gamma_1 : k.small_pressure / (k.gamma - 1.0);
  P.tvdlfeps = k.tvdlfeps;
  P.cada3_radius = k.cada3_radius;
  for (int d = 0; d < 3; ++d) P.schmid_rad[d] = k.schmid_rad[d];
  P.schmid_global = k.schmid_global;
  P.glm_alpha = k.mhd_glm_alpha;
  P.divbdiff = k.divbdiff;
  P.courantpar = k.courantpar;
  P.limiter = k.limiter;
  P.boundspeed = k.typeboundspeed;
  P.divb = k.physics == 1 ? k.typedivbfix : 0;
  P.glm_extended = k.mhd_glm_extended;
  P.fix_small_values = k.fix_small_values;
  P.check_small_values = k.check_small_values;
  P.small_values_method = k.small_values_method;
  P.small_values_daverage = k.small_values_daverage;
  // physical boundaries: per side all variables periodic, all cont, or all symm/asymm
  for (int s = 0; s < 6; ++s) {
    c->bc.kind[s] = 0;
    c->bc.flip[s] = 0;
    if (s >= 2 * k.ndim) continue;
    int per = 0, cont = 0, mir = 0;
    for (int v = 0; v < nw; ++v) {
      const int t = k.typeboundary[s][v];
      if (t == AMRVAC_BC_PERIODIC) ++per;
      else if (t == AMRVAC_BC_CONT) ++cont;
      else if (t == AMRVAC_BC_SYMM || t == AMRVAC_BC_ASYMM) {
        ++mir;
        if (t == AMRVAC_BC_ASYMM) c->bc.flip[s] |= 1u << v;
      } else {
        delete c;
        return fail(AMRVAC_E_UNSUPPORTED, "typeboundary must be periodic, cont, symm or asymm");
      }
    }
    if (per == nw) c->bc.kind[s] = BCK_PERIODIC;
    else if (cont == nw) c->bc.kind[s] = BCK_CONT;
    else if (mir == nw) c->bc.kind[s] = BCK_MIRROR;
    else {
      delete c;
      return fail(AMRVAC_E_UNSUPPORTED, "mixed boundary kinds on one side");
    }
  }
  for (int d = 0; d < 3; ++d) {
    if (d < k.ndim) {
      srl_maps_1d(k.nghostcells, bn, c->maps.smin[d], c->maps.smax[d], c->maps.rmin[d], c->maps.rmax[d]);
    } else {
      for (int q = 0; q < 3; ++q) c->maps.smin[d][q] = c->maps.smax[d][q] = c->maps.rmin[d][q] = c->maps.rmax[d][q] = 0;
    }
  }
  if ((e0 = c->ks.prepare()) != cudaSuccess) {
    delete c;
    return cuda_fail(e0, "cudaFuncSetAttribute");
  }
  for (int v = 1; v < c->ks.nvar; ++v) {
    if ((e0 = c->ks.prepare_v[v]()) != cudaSuccess) {
      delete c;
      return cuda_fail(e0, "cudaFuncSetAttribute");
    }
  }
  c->zchunk = valid_zchunk(bn, k.zchunk) ? k.zchunk : 0;
  {
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    c->wave_ctas = nsm * c->ks.ctas_per_sm();
    for (int v = 0; v < c->ks.nvar; ++v) c->wave_v[v] = nsm * c->ks.ctas_v[v]();
  }
  c->per_block = 1;
  for (int d = 0; d < k.ndim; ++d) c->per_block *= bn;
  cudaError_t e;
  if ((e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking)) != cudaSuccess) {
    delete c;
    return cuda_fail(e, "cudaStreamCreate");
  }
  // scalars: dt, cmax_global, time, time_max, dtsave, dtmin, courantpar, final
  // flag, slowsteps, steps since set_time, a2max_global(1:3) (schmid1)
  const double sc[13] = {0.0, 0.0, 0.0, 1.0e99, 0.0, k.dtmin, k.courantpar, 0.0, double(k.slowsteps), 0.0,
                         0.0, 0.0, 0.0};
  if ((e = cudaMalloc(&c->d_scal, sizeof(sc))) != cudaSuccess ||
      (e = cudaMemcpy(c->d_scal, sc, sizeof(sc), cudaMemcpyHostToDevice)) != cudaSuccess ||
      (e = cudaMalloc(&c->d_red, 2 * sizeof(unsigned long long))) != cudaSuccess ||
      (e = cudaMemset(c->d_red, 0, 2 * sizeof(unsigned long long))) != cudaSuccess ||
      (e = cudaMalloc(&c->d_status, sizeof(uint32_t))) != cudaSuccess ||
      (e = cudaMemset(c->d_status, 0, sizeof(uint32_t))) != cudaSuccess) {
    amrvac_gpu_destroy(c);
    return cuda_fail(e, "context allocation");
  }
  if (c->sv_on) {
    // per CTA: five [nw][(bn+4)^ndim] arrays and two flag arrays; as many
    // CTAs as fit in 256 MB, at most one per SM
    size_t gc = 1;
    for (int d = 0; d < k.ndim; ++d) gc *= (size_t)(bn + 4);
    c->sv_per_cta = 5 * (size_t)nw * gc + (2 * gc + 7) / 8;
    int nsm = 148, dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const size_t fit = ((size_t)256 << 20) / (sizeof(double) * c->sv_per_cta);
    c->sv_ctas = (int)std::max<size_t>(1, std::min<size_t>(fit, (size_t)nsm));
    if ((e = cudaMalloc(&c->sv_scratch, sizeof(double) * c->sv_per_cta * c->sv_ctas)) != cudaSuccess) {
      amrvac_gpu_destroy(c);
      return cuda_fail(e, "small-value scratch allocation");
    }
  }
  *out = c;
  return 0;
}

int amrvac_gpu_destroy(amrvac_ctx *c) {
  if (!c) return AMRVAC_E_ARG;
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->graph) cudaGraphExecDestroy(c->graph);
  for (int r = 0; r < 4; ++r) cudaFree(c->pool[r]);
  cudaFree(c->d_nbr);
  cudaFree(c->d_dx);
  cudaFree(c->d_scal);
  cudaFree(c->d_red);
  cudaFree(c->d_status);
  cudaFree(c->d_block_status);
  for (int r = 0; r < 3; ++r) cudaFree(c->d_adj[r]);
  cudaFree(c->d_amr_int);
  cudaFree(c->d_amr_err);
  cudaFree(c->d_stage);
  cudaFree(c->sv_scratch);
  cudaFree(c->sv_snap);
  delete c->amr;
  cudaFree(c->amr_gbuf);
  cudaFree(c->amr_pflux);
  cudaFree(c->amr_bxmin);
  cudaFree(c->amr_ints);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return 0;
}

static int set_blocks_impl(amrvac_ctx *c, int nblocks, const double *dx, const int *neighbor, bool level_jumps,
                           double *adopt_reg0 = nullptr);

int amrvac_gpu_set_blocks(amrvac_ctx *c, int nblocks, const double *dx, const int *neighbor) {
  if (c) c->a2max_set = false;
  return set_blocks_impl(c, nblocks, dx, neighbor, false);
}

// neighbor entries: block id, -1 physical boundary, and (multi-level grids,
// internal) <= -2 for a level jump whose ghost cells come from the ghost pass.
// adopt_reg0: a device buffer of nblocks blocks that becomes register 0 (the
// state after a regrid) instead of a zeroed one; it is the caller's to free
// unless c->pool[0] == adopt_reg0 afterwards.
static int set_blocks_impl(amrvac_ctx *c, int nblocks, const double *dx, const int *neighbor, bool level_jumps,
                           double *adopt_reg0) {
  if (int r = check_ctx(c, false)) return r;
  if (nblocks <= 0 || !dx || !neighbor) return fail(AMRVAC_E_ARG, "bad block description");
  const int nd = c->cfg.ndim;
  int ndir3 = 1;
  for (int d = 0; d < nd; ++d) ndir3 *= 3;
  std::vector<int> nbr((size_t)nblocks * 27, -1);
  std::vector<double> dxb((size_t)nblocks * 3, 1.0);
  for (int b = 0; b < nblocks; ++b) {
    for (int q = 0; q < ndir3; ++q) {
      const int di = q % 3 - 1, dj = nd >= 2 ? (q / 3) % 3 - 1 : 0, dk = nd >= 3 ? q / 9 - 1 : 0;
      const int v = neighbor[(size_t)b * ndir3 + q];
      if (v >= nblocks || (v < -1 && !level_jumps)) return fail(AMRVAC_E_ARG, "neighbor id out of range");
      nbr[(size_t)b * 27 + (di + 1) + 3 * (dj + 1) + 9 * (dk + 1)] = v;
    }
    nbr[(size_t)b * 27 + 13] = b;
    for (int d = 0; d < nd; ++d) {
      const double h = dx[(size_t)b * nd + d];
      if (!(h > 0.0)) return fail(AMRVAC_E_ARG, "dx must be positive");
      dxb[(size_t)b * 3 + d] = h;
    }
  }
  // a physical side needs a boundary kind, a sibling side must not be marked
  for (int b = 0; b < nblocks; ++b)
    for (int d = 0; d < nd; ++d)
      for (int s = 0; s < 2; ++s) {
        int o[3] = {0, 0, 0};
        o[d] = s ? 1 : -1;
        const int v = nbr[(size_t)b * 27 + (o[0] + 1) + 3 * (o[1] + 1) + 9 * (o[2] + 1)];
        if (v == -1 && c->bc.kind[2 * d + s] == BCK_PERIODIC)
          return fail(AMRVAC_E_ARG, "physical boundary on a side declared periodic");
      }
  // every direction whose face components all lead to siblings must exist
  for (int b = 0; b < nblocks; ++b)
    for (int q = 0; q < 27; ++q) {
      const int o[3] = {q % 3 - 1, (q / 3) % 3 - 1, q / 9 - 1};
      bool inner = true, any = false;
      for (int d = 0; d < 3; ++d) {
        if (!o[d]) continue;
        if (d >= nd) { inner = false; break; }
        any = true;
        int f[3] = {0, 0, 0};
        f[d] = o[d];
        if (nbr[(size_t)b * 27 + (f[0] + 1) + 3 * (f[1] + 1) + 9 * (f[2] + 1)] < 0) inner = false;
      }
      if (any && inner && nbr[(size_t)b * 27 + q] == -1)
        return fail(AMRVAC_E_ARG, "missing edge/corner neighbour between two sibling faces");
    }
  cudaStreamSynchronize(c->stream);
  if (c->graph) { cudaGraphExecDestroy(c->graph); c->graph = nullptr; }
  const size_t bytes = sizeof(double) * c->per_block * c->nw * nblocks;
  if (adopt_reg0 && adopt_reg0 == c->pool[1]) {
    // regrid into the scratch register: swap it in, nothing is allocated
    std::swap(c->pool[0], c->pool[1]);
  } else if (adopt_reg0) {
    // regrid into a new, larger buffer: the other registers follow its size
    const size_t cap = (size_t)nblocks + nblocks / 4 + 1;
    for (int r = 0; r < 4; ++r) { cudaFree(c->pool[r]); c->pool[r] = nullptr; }
    c->pool_cap = 0;
    c->pool[0] = adopt_reg0;
    for (int r = 1; r < c->nreg; ++r) CK(cudaMalloc(&c->pool[r], sizeof(double) * c->per_block * c->nw * cap));
    c->pool_cap = cap;
  } else {
    if ((size_t)nblocks > c->pool_cap || !c->pool[0]) {
      for (int r = 0; r < 4; ++r) { cudaFree(c->pool[r]); c->pool[r] = nullptr; }
      c->pool_cap = 0;
      const size_t cap = (size_t)nblocks + nblocks / 4 + 1;
      for (int r = 0; r < c->nreg; ++r) CK(cudaMalloc(&c->pool[r], sizeof(double) * c->per_block * c->nw * cap));
      c->pool_cap = cap;
      if (c->sv_on) {
        cudaFree(c->sv_snap);
        c->sv_snap = nullptr;
        CK(cudaMalloc(&c->sv_snap, sizeof(double) * c->per_block * c->nw * cap));
      }
    }
    for (int r = 0; r < c->nreg; ++r) CK(cudaMemsetAsync(c->pool[r], 0, bytes, c->stream));
  }
  c->nblocks = nblocks;
  if ((size_t)nblocks > c->nbr_cap || !c->d_nbr) {
    cudaFree(c->d_nbr); cudaFree(c->d_dx); cudaFree(c->d_block_status);
    c->d_nbr = nullptr; c->d_dx = nullptr; c->d_block_status = nullptr;
    c->nbr_cap = 0;
    const size_t cap = (size_t)nblocks + nblocks / 4 + 1;
    CK(cudaMalloc(&c->d_nbr, sizeof(int) * 27 * cap));
    CK(cudaMalloc(&c->d_dx, sizeof(double) * 3 * cap));
    CK(cudaMalloc(&c->d_block_status, sizeof(uint32_t) * cap));
    c->nbr_cap = cap;
  }
  CK(cudaMemcpyAsync(c->d_nbr, nbr.data(), sizeof(int) * nbr.size(), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->d_dx, dxb.data(), sizeof(double) * dxb.size(), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemsetAsync(c->d_block_status, 0, sizeof(uint32_t) * nblocks, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->h_dx = dxb;
  for (int r = 0; r < 3; ++r) { cudaFree(c->d_adj[r]); c->d_adj[r] = nullptr; }
  c->adj_prepared = false;
  delete c->amr; c->amr = nullptr;
  return 0;
}

int amrvac_gpu_set_uniform_grid(amrvac_ctx *c, const int *domain_nx, const double *xprobmin,
                                const double *xprobmax) {
  if (int r = check_ctx(c, false)) return r;
  if (!domain_nx || !xprobmin || !xprobmax) return fail(AMRVAC_E_ARG, "null argument");
  const int nd = c->cfg.ndim;
  int nb[3] = {1, 1, 1};
  double h[3] = {1, 1, 1};
  int total = 1;
  for (int d = 0; d < nd; ++d) {
    if (domain_nx[d] <= 0 || domain_nx[d] % c->bn) return fail(AMRVAC_E_ARG, "domain_nx must be a multiple of block_nx");
    nb[d] = domain_nx[d] / c->bn;
    h[d] = (xprobmax[d] - xprobmin[d]) / double(domain_nx[d]);
    total *= nb[d];
  }
  int ndir3 = 1;
  for (int d = 0; d < nd; ++d) ndir3 *= 3;
  std::vector<int> nbr((size_t)total * ndir3);
  std::vector<double> dx((size_t)total * nd);
  for (int b = 0; b < total; ++b) {
    const int ig[3] = {b % nb[0], (b / nb[0]) % nb[1], b / (nb[0] * nb[1])};
    for (int q = 0; q < ndir3; ++q) {
      const int o[3] = {q % 3 - 1, nd >= 2 ? (q / 3) % 3 - 1 : 0, nd >= 3 ? q / 9 - 1 : 0};
      int jg[3] = {0, 0, 0};
      bool ok = true;
      for (int d = 0; d < nd; ++d) {
        jg[d] = ig[d] + o[d];
        if (jg[d] < 0 || jg[d] >= nb[d]) {
          const int side = jg[d] < 0 ? 0 : 1;
          if (c->bc.kind[2 * d + side] == BCK_PERIODIC) jg[d] = (jg[d] + nb[d]) % nb[d];
          else ok = false;
        }
      }
      nbr[(size_t)b * ndir3 + q] = ok ? jg[0] + nb[0] * (jg[1] + nb[1] * jg[2]) : -1;
    }
    for (int d = 0; d < nd; ++d) dx[(size_t)b * nd + d] = h[d];
  }
  return amrvac_gpu_set_blocks(c, total, dx.data(), nbr.data());
}

// A static multi-level grid: leaf blocks (level, ig) of a 2:1 balanced tree
// over a periodic domain of nbase root blocks per direction (the reference's
// forest, src/amr/mod_forest.t, with the neighbour kinds of
// src/amr/mod_amr_neighbors.t: sibling, coarser, finer).  Same-level ghost
// cells are read through the neighbour table as on a uniform grid; the ghost
// cells of every level-jump direction are written by the ghost pass before
// each stage, and every stage ends with fix_conserve.
static int amr_grid_impl(amrvac_ctx *c, int nleaf, const int *leaf, const int *nbase, const double *xprobmin,
                         const double *xprobmax, const int *ops);

int amrvac_gpu_set_amr_grid(amrvac_ctx *c, int nleaf, const int *leaf, const int *nbase, const double *xprobmin,
                            const double *xprobmax) {
  return amr_grid_impl(c, nleaf, leaf, nbase, xprobmin, xprobmax, nullptr);
}

// Regrid in place (amr_coarsen_refine): the new leaves and, per new leaf, how
// its state comes from the old tree's register 0 (see AmrRemapArgs).  The
// domain and root blocks stay those of the current grid; registers 1 and 2
// are scratch afterwards.
int amrvac_gpu_amr_regrid(amrvac_ctx *c, int nleaf, const int *leaf, const int *op) {
  if (c) c->a2max_set = false;
  if (int r = check_ctx(c, true)) return r;
  if (!c->amr) return fail(AMRVAC_E_STATE, "amr_regrid: no multi-level grid (amrvac_gpu_set_amr_grid)");
  if (!op) return fail(AMRVAC_E_ARG, "amr_regrid: null op table");
  int nbase[3];
  double xmin[3], xmax[3];
  for (int d = 0; d < 3; ++d) {
    nbase[d] = c->amr->nbase[d];
    xmin[d] = c->amr->xmin[d];
    xmax[d] = c->amr->xmax[d];
  }
  return amr_grid_impl(c, nleaf, leaf, nbase, xmin, xmax, op);
}

static int amr_grid_impl(amrvac_ctx *c, int nleaf, const int *leaf, const int *nbase, const double *xprobmin,
                         const double *xprobmax, const int *ops) {
  if (int r = check_ctx(c, false)) return r;
  const int nd = c->cfg.ndim;
  if (nleaf <= 0 || !leaf || !nbase || !xprobmin || !xprobmax) return fail(AMRVAC_E_ARG, "set_amr_grid: bad arguments");
  if (nd < 2) return fail(AMRVAC_E_UNSUPPORTED, "set_amr_grid: ndim 2 or 3");
  if (c->sv_on) return fail(AMRVAC_E_UNSUPPORTED, "set_amr_grid: not with small_values_method average");
  if (c->cfg.nghostcells != 2) return fail(AMRVAC_E_UNSUPPORTED, "set_amr_grid: nghostcells 2");
  bool periodic[3] = {true, true, true};
  for (int d = 0; d < nd; ++d) {
    const bool p0 = c->bc.kind[2 * d] == BCK_PERIODIC, p1 = c->bc.kind[2 * d + 1] == BCK_PERIODIC;
    if (p0 != p1) return fail(AMRVAC_E_ARG, "set_amr_grid: a dimension is periodic on one side only");
    periodic[d] = p0;
  }
  int maxlev = 1;
  for (int b = 0; b < nleaf; ++b) {
    const int L = leaf[4 * b];
    if (L < 1 || L > AMR_MAX_LEVELS) return fail(AMRVAC_E_ARG, "set_amr_grid: level out of range");
    maxlev = std::max(maxlev, L);
  }
  // dense owner maps per level: leaf id, -2 refined, -1 covered by a coarser
  // leaf, -3 not covered
  AmrGhostArgs G;
  std::memset(&G, 0, sizeof(G));
  size_t total = 0;
  for (int L = 1; L <= maxlev; ++L) {
    size_t n = 1;
    for (int d = 0; d < 3; ++d) {
      G.nlev[L][d] = d < nd ? (nbase[d] << (L - 1)) : 1;
      if (d < nd && nbase[d] <= 0) return fail(AMRVAC_E_ARG, "set_amr_grid: nbase must be positive");
      n *= (size_t)G.nlev[L][d];
    }
    G.owner_off[L] = (int)total;
    total += n;
    if (total > ((size_t)1 << 26)) return fail(AMRVAC_E_UNSUPPORTED, "set_amr_grid: hierarchy too deep for the owner maps");
  }
  std::vector<int> owner(total, -3);
  auto at = [&](int L, const int *jg) -> int & {
    return owner[(size_t)G.owner_off[L] + jg[0] + (size_t)G.nlev[L][0] * (jg[1] + (size_t)G.nlev[L][1] * jg[2])];
  };
  std::vector<int> lev(nleaf), ig(3 * (size_t)nleaf, 0);
  for (int b = 0; b < nleaf; ++b) {
    const int L = leaf[4 * b];
    lev[b] = L;
    int g[3] = {0, 0, 0};
    for (int d = 0; d < nd; ++d) {
      g[d] = leaf[4 * b + 1 + d];
      if (g[d] < 0 || g[d] >= G.nlev[L][d]) return fail(AMRVAC_E_ARG, "set_amr_grid: block index out of range");
      ig[3 * b + d] = g[d];
    }
    if (at(L, g) != -3) return fail(AMRVAC_E_ARG, "set_amr_grid: overlapping leaves");
    at(L, g) = b;
    for (int L2 = L - 1; L2 >= 1; --L2) {  // ancestors are refined
      int a[3] = {0, 0, 0};
      for (int d = 0; d < nd; ++d) a[d] = g[d] >> (L - L2);
      int &o = at(L2, a);
      if (o >= 0 || o == -1) return fail(AMRVAC_E_ARG, "set_amr_grid: overlapping leaves");
      o = -2;
    }
  }
  for (int b = 0; b < nleaf; ++b)  // descendants are covered
    for (int L2 = lev[b] + 1; L2 <= maxlev; ++L2) {
      const int f = 1 << (L2 - lev[b]);
      const int fy = nd >= 2 ? f : 1, fz = nd >= 3 ? f : 1;
      for (int z = 0; z < fz; ++z)
        for (int y = 0; y < fy; ++y)
          for (int x = 0; x < f; ++x) {
            const int g[3] = {ig[3 * b] * f + x, nd >= 2 ? ig[3 * b + 1] * f + y : 0, nd >= 3 ? ig[3 * b + 2] * f + z : 0};
            int &o = at(L2, g);
            if (o != -3) return fail(AMRVAC_E_ARG, "set_amr_grid: overlapping leaves");
            o = -1;
          }
    }
  for (int L = 1; L <= maxlev; ++L)  // every region is covered
    for (int z = 0; z < G.nlev[L][2]; ++z)
      for (int y = 0; y < G.nlev[L][1]; ++y)
        for (int x = 0; x < G.nlev[L][0]; ++x) {
          const int g[3] = {x, y, z};
          const int o = at(L, g);
          if (o == -3) {
            const int p[3] = {x / 2, y / 2, z / 2};
            if (L == 1 || at(L - 1, p) == -2) return fail(AMRVAC_E_ARG, "set_amr_grid: leaves do not cover the domain");
          }
          if (o == -2 && L == maxlev) return fail(AMRVAC_E_ARG, "set_amr_grid: inconsistent tree");
        }
  // neighbour kinds, the neighbour table and the children across each face
  const int nb = nleaf;
  std::vector<int> ntype(27 * (size_t)nb, AMR_BOUNDARY), child(27 * 8 * (size_t)nb, -1);
  std::vector<int> gslot(nb, -1), face(nb, 0), iblocks;
  int ndir3 = 1;
  for (int d = 0; d < nd; ++d) ndir3 *= 3;
  std::vector<int> nbr((size_t)nb * ndir3, -1);
  std::vector<double> dx((size_t)nb * nd), bxmin(3 * (size_t)nb, 0.0), dxb3(3 * (size_t)nb, 1.0);
  for (int b = 0; b < nb; ++b) {
    const int L = lev[b];
    for (int q = 0; q < 27; ++q) {
      const int dd[3] = {q % 3 - 1, (q / 3) % 3 - 1, q / 9 - 1};
      bool ok = true;
      int jg[3] = {0, 0, 0};
      for (int d = 0; d < 3; ++d) {
        if (d >= nd) { if (dd[d]) ok = false; continue; }
        const int nl = G.nlev[L][d];
        const int j = ig[3 * b + d] + dd[d];
        if ((j < 0 || j >= nl) && !periodic[d]) ok = false;  // a physical boundary
        jg[d] = (j % nl + nl) % nl;
      }
      if (!ok) continue;
      if (q == 13) { ntype[b * 27 + q] = AMR_SIBLING; continue; }
      const int o = at(L, jg);
      if (o >= 0) {
        ntype[b * 27 + q] = AMR_SIBLING;
      } else if (o == -1) {
        const int p[3] = {jg[0] / 2, jg[1] / 2, jg[2] / 2};
        if (L == 1 || at(L - 1, p) < 0) return fail(AMRVAC_E_ARG, "set_amr_grid: tree not 2:1 balanced");
        ntype[b * 27 + q] = AMR_COARSE;
      } else {
        ntype[b * 27 + q] = AMR_FINE;
        for (int cb = 0; cb < (1 << nd); ++cb) {
          const int cc[3] = {cb & 1, (cb >> 1) & 1, (cb >> 2) & 1};
          bool adjacent = true;
          for (int d = 0; d < nd; ++d)
            if ((dd[d] == 1 && cc[d] != 0) || (dd[d] == -1 && cc[d] != 1)) adjacent = false;
          const int g2[3] = {2 * jg[0] + cc[0], nd >= 2 ? 2 * jg[1] + cc[1] : 0, nd >= 3 ? 2 * jg[2] + cc[2] : 0};
          const int o2 = at(L + 1, g2);
          if (adjacent && o2 < 0) return fail(AMRVAC_E_ARG, "set_amr_grid: tree not 2:1 balanced");
          child[(b * 27 + q) * 8 + cb] = o2 >= 0 ? o2 : -1;
        }
      }
    }
    bool jump = false;
    for (int q = 0; q < 27; ++q) jump |= ntype[b * 27 + q] == AMR_COARSE || ntype[b * 27 + q] == AMR_FINE;
    if (jump) {
      gslot[b] = (int)iblocks.size();
      iblocks.push_back(b);
    }
    for (int d = 0; d < nd; ++d)
      for (int s = 0; s < 2; ++s) {
        int o[3] = {0, 0, 0};
        o[d] = s ? 1 : -1;
        const int t = ntype[b * 27 + (o[0] + 1) + 3 * (o[1] + 1) + 9 * (o[2] + 1)];
        if (t == AMR_COARSE || t == AMR_FINE) face[b] |= 1 << (2 * d + s);
      }
    for (int d = 0; d < nd; ++d) {
      // cell size and corner as the reference's block geometry computes them
      const double h = (xprobmax[d] - xprobmin[d]) / (nbase[d] * double(c->bn) * double(1 << (L - 1)));
      dx[(size_t)b * nd + d] = h;
      dxb3[3 * (size_t)b + d] = h;
      bxmin[3 * (size_t)b + d] = xprobmin[d] + ig[3 * b + d] * double(c->bn) * h;
    }
  }
  for (int b = 0; b < nb; ++b)
    for (int q = 0; q < ndir3; ++q) {
      const int dd[3] = {q % 3 - 1, nd >= 2 ? (q / 3) % 3 - 1 : 0, nd >= 3 ? q / 9 - 1 : 0};
      const int q27 = (dd[0] + 1) + 3 * (dd[1] + 1) + 9 * (dd[2] + 1);
      const int t = ntype[b * 27 + q27];
      if (t == AMR_BOUNDARY) {
        nbr[(size_t)b * ndir3 + q] = -1;
      } else if (t == AMR_SIBLING) {
        int jg[3] = {0, 0, 0};
        for (int d = 0; d < nd; ++d) {
          const int nl = G.nlev[lev[b]][d];
          jg[d] = ((ig[3 * b + d] + dd[d]) % nl + nl) % nl;
        }
        nbr[(size_t)b * ndir3 + q] = q27 == 13 ? b : at(lev[b], jg);
      } else {
        nbr[(size_t)b * ndir3 + q] = -2 - gslot[b];
      }
    }
  // regrid: build the new register 0 from the old tree before it goes away
  double *newreg = nullptr;
  if (ops) {
    const int nold = c->nblocks, nch = 1 << nd;
    const std::vector<int> &old_leaf = c->amr->h_leaf;
    auto same_block = [&](int ob, int L, const int *g) {
      if (old_leaf[4 * ob] != L) return false;
      for (int d = 0; d < nd; ++d)
        if (old_leaf[4 * ob + 1 + d] != g[d]) return false;
      return true;
    };
    for (int b = 0; b < nb; ++b) {
      const int *o = ops + 9 * (size_t)b;
      const int L = lev[b];
      const int *g = &ig[3 * b];
      bool ok = true;
      if (o[0] == 0) {
        ok = o[1] >= 0 && o[1] < nold && same_block(o[1], L, g);
      } else if (o[0] == 1) {
        int pg[3] = {0, 0, 0}, cb = 0;
        for (int d = 0; d < nd; ++d) {
          pg[d] = g[d] >> 1;
          cb |= (g[d] & 1) << d;
        }
        ok = o[1] >= 0 && o[1] < nold && o[2] == cb && L > 1 && same_block(o[1], L - 1, pg);
      } else if (o[0] == 2) {
        for (int q = 0; q < nch && ok; ++q) {
          int cg[3] = {0, 0, 0};
          for (int d = 0; d < nd; ++d) cg[d] = 2 * g[d] + ((q >> d) & 1);
          ok = o[1 + q] >= 0 && o[1 + q] < nold && same_block(o[1 + q], L + 1, cg);
        }
      } else {
        ok = false;
      }
      if (!ok) return fail(AMRVAC_E_ARG, "amr_regrid: op " + std::to_string(b) + " does not match the old and new trees");
    }
    if (int r = launch_amr_ghost_pass(c, 0)) return r;  // the old tree's level-jump ghosts
    int *d_op = nullptr;
    cudaError_t e = cudaSuccess;
    if ((size_t)nb <= c->pool_cap) newreg = c->pool[1];  // scratch register: swapped in afterwards
    else e = cudaMalloc(&newreg, sizeof(double) * c->per_block * c->nw * ((size_t)nb + nb / 4 + 1));
    if (e == cudaSuccess) e = cudaMalloc(&d_op, sizeof(int) * 9 * (size_t)nb);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(d_op, ops, sizeof(int) * 9 * (size_t)nb, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) {
      AmrRemapArgs R;
      std::memset(&R, 0, sizeof(R));
      R.old = stage_args(c, 0, 0, 0, 0.0, 1.0, 1.0);
      R.op = d_op;
      R.unew = newreg;
      R.nw = c->nw;
      e = launch_amr_remap(R, nb, nd, c->stream);
      ++c->launches;
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    cudaFree(d_op);
    if (e != cudaSuccess) {
      if (newreg != c->pool[1]) cudaFree(newreg);
      return cuda_fail(e, "amr_regrid");
    }
  }
  if (int r = set_blocks_impl(c, nb, dx.data(), nbr.data(), true, newreg)) {
    if (newreg && c->pool[0] != newreg && c->pool[1] != newreg) cudaFree(newreg);
    return r;
  }
  // device copies
  AmrDev *A = new AmrDev();
  c->amr = A;
  A->h_leaf.assign(4 * (size_t)nb, 0);
  for (int b = 0; b < nb; ++b) {
    A->h_leaf[4 * b] = lev[b];
    for (int d = 0; d < nd; ++d) A->h_leaf[4 * b + 1 + d] = ig[3 * b + d];
  }
  for (int d = 0; d < 3; ++d) {
    A->nbase[d] = d < nd ? nbase[d] : 1;
    A->xmin[d] = d < nd ? xprobmin[d] : 0.0;
    A->xmax[d] = d < nd ? xprobmax[d] : 1.0;
  }
  A->nslots = (int)iblocks.size();
  const size_t ns = std::max<size_t>(1, iblocks.size());
  std::vector<int> ints;
  auto put = [&](const std::vector<int> &v) {
    const size_t off = ints.size();
    ints.insert(ints.end(), v.begin(), v.end());
    return off;
  };
  const size_t o_ib = put(iblocks), o_gs = put(gslot), o_fc = put(face), o_nt = put(ntype), o_lv = put(lev),
               o_ig = put(ig), o_ch = put(child), o_ow = put(owner);
  CK(ensure_capacity(&c->amr_ints, &c->amr_ints_cap, ints.size()));
  A->d_int = c->amr_ints;
  CK(cudaMemcpyAsync(A->d_int, ints.data(), sizeof(int) * ints.size(), cudaMemcpyHostToDevice, c->stream));
  CK(ensure_capacity(&c->amr_bxmin, &c->amr_bxmin_cap, bxmin.size()));
  A->d_bxmin = c->amr_bxmin;
  CK(cudaMemcpyAsync(A->d_bxmin, bxmin.data(), sizeof(double) * bxmin.size(), cudaMemcpyHostToDevice, c->stream));
  size_t gcells = 1;
  for (int d = 0; d < nd; ++d) gcells *= (size_t)c->bn + 4;
  // every ghost cell a kernel reads is written by the ghost pass first, and
  // every face flux the fix reads by the stage before it: no clearing needed
  CK(ensure_capacity(&c->amr_gbuf, &c->amr_gbuf_cap, ns * c->nw * gcells));
  A->gbuf = c->amr_gbuf;
  CK(ensure_capacity(&c->amr_pflux, &c->amr_pflux_cap, ns * 2 * nd * c->nw * (size_t)c->bn * c->bn));
  A->pflux = c->amr_pflux;
  A->d_gslot = A->d_int + o_gs;
  A->d_face = A->d_int + o_fc;
  G.u = nullptr;
  G.gbuf = A->gbuf;
  G.nw = c->nw;
  G.iblocks = A->d_int + o_ib;
  G.ntype = A->d_int + o_nt;
  G.level = A->d_int + o_lv;
  G.ig = A->d_int + o_ig;
  G.bxmin = A->d_bxmin;
  G.dxb = c->d_dx;
  G.owner = A->d_int + o_ow;
  G.maxlevel = maxlev;
  G.bn = c->bn;
  for (int q = 0; q < 6; ++q) {
    G.bc_kind[q] = c->bc.kind[q];
    G.bc_flip[q] = c->bc.flip[q];
  }
  G.status = c->d_status;
  A->G = G;
  CK(prepare_amr_ghosts(nd, c->bn));
  std::memset(&A->F, 0, sizeof(A->F));
  A->F.pflux = A->pflux;
  A->F.nw = c->nw;
  A->F.bn = c->bn;
  A->F.iblocks = G.iblocks;
  A->F.gslot = A->d_gslot;
  A->F.ntype = G.ntype;
  A->F.child = A->d_int + o_ch;
  A->F.sweep = -1;
  A->F.scal = c->d_scal;
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

int amrvac_gpu_amr_slots(const amrvac_ctx *c) { return c && c->amr ? c->amr->nslots : 0; }

int amrvac_gpu_amr_leaves(const amrvac_ctx *c, int *leaf) {
  if (!c || !c->amr) return AMRVAC_E_STATE;
  if (leaf) std::memcpy(leaf, c->amr->h_leaf.data(), sizeof(int) * c->amr->h_leaf.size());
  return (int)(c->amr->h_leaf.size() / 4);
}

// resettree (src/amr/mod_amr_grid.t:45-73): errest with the Löhner estimator
// on register 0, the tree decision of amr_coarsen_refine (amrvac_amr_plan, on
// the host), and the device remap; *changed = 0 when the tree stays.
int amrvac_gpu_amr_resettree(amrvac_ctx *c, const double *weight, const int *logflag, int refine_max_level,
                             const double *refine_threshold, const double *derefine_ratio,
                             const double *amr_wavefilter, int *changed) {
  if (int r = check_ctx(c, true)) return r;
  if (!c->amr) return fail(AMRVAC_E_STATE, "amr_resettree: no multi-level grid (amrvac_gpu_set_amr_grid)");
  const int nb = c->nblocks, nd = c->cfg.ndim;
  std::vector<int> lev(nb), flags(nb);
  for (int b = 0; b < nb; ++b) lev[b] = c->amr->h_leaf[4 * b];
  if (int r = amrvac_gpu_lohner(c, 0, weight, logflag, refine_max_level, refine_threshold, derefine_ratio,
                                amr_wavefilter, lev.data(), flags.data(), nullptr))
    return r;
  std::vector<unsigned char> ref(nb), coa(nb);
  bool any = false;
  for (int b = 0; b < nb; ++b) {
    ref[b] = (flags[b] & 1) != 0;
    coa[b] = (flags[b] & 2) != 0;
    any = any || ref[b] || coa[b];
  }
  if (!any) {  // nothing to refine or coarsen: the tree stays (it is 2:1 balanced)
    if (changed) *changed = 0;
    return 0;
  }
  const std::vector<int> old_leaf = c->amr->h_leaf;
  const int cap = nb * (1 << nd);
  std::vector<int> leaf_new(4 * (size_t)cap), op(9 * (size_t)cap);
  int nnew = 0;
  int periodic[3] = {1, 1, 1};
  for (int d = 0; d < nd; ++d) periodic[d] = c->bc.kind[2 * d] == BCK_PERIODIC;
  if (int r = amrvac_amr_plan(nd, c->amr->nbase, periodic, refine_max_level, nb, old_leaf.data(), ref.data(), coa.data(), cap,
                              &nnew, leaf_new.data(), op.data()))
    return fail(r, "amr_resettree: tree decision failed");
  leaf_new.resize(4 * (size_t)nnew);
  const bool same = nnew == nb && leaf_new == old_leaf;
  if (changed) *changed = same ? 0 : 1;
  if (same) return 0;
  return amrvac_gpu_amr_regrid(c, nnew, leaf_new.data(), op.data());
}

// Average device time of the level-jump ghost pass (on register 0) and of the
// flux fix (on register 2, whose contents it changes) over reps launches.
int amrvac_gpu_amr_kernel_ms(amrvac_ctx *c, int reps, double *ghost_ms, double *fix_ms) {
  if (int r = check_ctx(c, true)) return r;
  if (!c->amr) return fail(AMRVAC_E_STATE, "amr_kernel_ms: no multi-level grid");
  if (reps <= 0 || !ghost_ms || !fix_ms) return fail(AMRVAC_E_ARG, "amr_kernel_ms: bad arguments");
  cudaEvent_t e[3];
  for (auto &x : e) CK(cudaEventCreate(&x));
  AmrFixArgs F = c->amr->F;
  F.w = c->pool[2];
  if (int r = launch_amr_ghost_pass(c, 0)) return r;  // warm
  CK(cudaEventRecord(e[0], c->stream));
  for (int i = 0; i < reps; ++i)
    if (int r = launch_amr_ghost_pass(c, 0)) return r;
  CK(cudaEventRecord(e[1], c->stream));
  for (int i = 0; i < reps; ++i) {
    CK(launch_amr_fix(F, c->amr->nslots, c->cfg.ndim, c->stream));
    ++c->launches;
  }
  CK(cudaEventRecord(e[2], c->stream));
  CK(cudaEventSynchronize(e[2]));
  float a, b;
  CK(cudaEventElapsedTime(&a, e[0], e[1]));
  CK(cudaEventElapsedTime(&b, e[1], e[2]));
  for (auto &x : e) cudaEventDestroy(x);
  *ghost_ms = a / reps;
  *fix_ms = b / reps;
  return 0;
}

int amrvac_gpu_nblocks(const amrvac_ctx *c) { return c ? c->nblocks : AMRVAC_E_ARG; }

static int ensure_stage(amrvac_ctx *c, size_t doubles) {
  if (c->stage_doubles >= doubles) return 0;
  cudaStreamSynchronize(c->stream);
  cudaFree(c->d_stage);
  c->d_stage = nullptr;
  c->stage_doubles = 0;
  CK(cudaMalloc(&c->d_stage, sizeof(double) * doubles));
  c->stage_doubles = doubles;
  return 0;
}

static size_t ghosted_per_block(const amrvac_ctx *c) {
  size_t g = 1;
  for (int d = 0; d < c->cfg.ndim; ++d) g *= (size_t)(c->bn + 2 * c->cfg.nghostcells);
  return g * c->nw;
}

int amrvac_gpu_upload(amrvac_ctx *c, int reg, int first, int n, const double *w) {
  if (int r = check_ctx(c, true)) return r;
  if (reg < 0 || reg > 2 || !w || first < 0 || n <= 0 || first + n > c->nblocks)
    return fail(AMRVAC_E_ARG, "bad upload range");
  const size_t gpb = ghosted_per_block(c);
  const int chunk = (int)std::max<size_t>(1, (size_t)(256u << 20) / (gpb * sizeof(double)));
  for (int b0 = 0; b0 < n; b0 += chunk) {
    const int m = std::min(chunk, n - b0);
    if (int r = ensure_stage(c, gpb * m)) return r;
    CK(cudaMemcpyAsync(c->d_stage, w + (size_t)b0 * gpb, sizeof(double) * gpb * m, cudaMemcpyHostToDevice,
                       c->stream));
    CK(launch_unpack(c->d_stage, c->pool[reg], first + b0, m, c->nw, c->cfg.ndim, c->cfg.nghostcells, c->bn,
                     c->stream));
    ++c->launches;
  }
  CK(cudaStreamSynchronize(c->stream));
  c->a2max_set = false;
  return 0;
}

int amrvac_gpu_download(amrvac_ctx *c, int reg, int first, int n, double *w) {
  if (int r = check_ctx(c, true)) return r;
  if (reg < 0 || reg > 2 || !w || first < 0 || n <= 0 || first + n > c->nblocks)
    return fail(AMRVAC_E_ARG, "bad download range");
  const size_t gpb = ghosted_per_block(c);
  const int chunk = (int)std::max<size_t>(1, (size_t)(256u << 20) / (gpb * sizeof(double)));
  for (int b0 = 0; b0 < n; b0 += chunk) {
    const int m = std::min(chunk, n - b0);
    if (int r = ensure_stage(c, gpb * m)) return r;
    if (c->amr && b0 == 0)
      if (int r = launch_amr_ghost_pass(c, reg)) return r;
    CK(launch_pack(c->pool[reg], c->d_stage, first + b0, m, c->nw, c->cfg.ndim, c->cfg.nghostcells, c->bn, c->d_nbr,
                   c->maps, c->bc, c->amr ? c->amr->gbuf : nullptr, c->stream));
    ++c->launches;
    CK(cudaMemcpyAsync(w + (size_t)b0 * gpb, c->d_stage, sizeof(double) * gpb * m, cudaMemcpyDeviceToHost,
                       c->stream));
    CK(cudaStreamSynchronize(c->stream));
  }
  return 0;
}

int amrvac_gpu_getdt(amrvac_ctx *c, int reg, double *dt, double *cmax_global) {
  if (int r = check_ctx(c, true)) return r;
  if (reg < 0 || reg > 2) return fail(AMRVAC_E_ARG, "bad register");
  if (int r = launch_getdt(c, reg)) return r;
  unsigned long long red[2];
  CK(cudaMemcpyAsync(red, c->d_red, sizeof(red), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemsetAsync(c->d_red, 0, sizeof(red), c->stream));
  CK(cudaStreamSynchronize(c->stream));
  double x, cm;
  std::memcpy(&x, &red[0], sizeof(double));
  std::memcpy(&cm, &red[1], sizeof(double));
  double d = 1.0e99;
  if (x > 1.0e-12) d = std::min(d, c->cfg.courantpar / x);
  if (dt) *dt = d;
  if (cmax_global) *cmax_global = cm;
  CK(cudaMemcpyAsync(c->d_scal + 1, &cm, sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return d < c->cfg.dtmin ? (int)AMRVAC_ST_DT_TOO_SMALL : 0;
}

int amrvac_gpu_set_cmax_global(amrvac_ctx *c, double cmax_global) {
  if (int r = check_ctx(c, false)) return r;
  CK(cudaMemcpyAsync(c->d_scal + 1, &cmax_global, sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

int amrvac_gpu_advect1(amrvac_ctx *c, int reg_ct, int reg_new, int reg_base, double a_base, double b_in,
                       double dtfactor, double dt) {
  if (int r = check_ctx(c, true)) return r;
  if (reg_ct < 0 || reg_ct > 2 || reg_new < 0 || reg_new > 2 || reg_base < 0 || reg_base > 2)
    return fail(AMRVAC_E_ARG, "bad register");
  if (reg_ct == reg_new) return fail(AMRVAC_E_ARG, "reg_ct and reg_new must differ");
  if (a_base == 0.0 && b_in != 1.0) return fail(AMRVAC_E_ARG, "a_base == 0 requires b_in == 1");
  if (int r = check_a2max(c)) return r;
  CK(cudaMemcpyAsync(c->d_scal + 0, &dt, sizeof(double), cudaMemcpyHostToDevice, c->stream));
  int r = launch_stage(c, reg_ct, reg_new, reg_base, a_base, b_in, dtfactor);
  CK(cudaStreamSynchronize(c->stream));
  return r;
}

int amrvac_gpu_advect1_dim(amrvac_ctx *c, int reg_ct, int reg_new, int reg_base, double a_base, double b_in,
                           double dtfactor, double dt, int idim) {
  if (int r = check_ctx(c, true)) return r;
  if (idim < 0 || idim > c->cfg.ndim) return fail(AMRVAC_E_ARG, "idim must be 0 (all) or 1..ndim");
  c->sweep = idim - 1;
  c->fixed_dir = idim > 0;
  const int r = amrvac_gpu_advect1(c, reg_ct, reg_new, reg_base, a_base, b_in, dtfactor, dt);
  c->sweep = -1;
  c->fixed_dir = false;
  return r;
}

int amrvac_gpu_set_time(amrvac_ctx *c, double t, double time_max, double dtsave) {
  if (int r = check_ctx(c, false)) return r;
  const double v[3] = {t, time_max, dtsave};
  CK(cudaMemcpyAsync(c->d_scal + 2, v, sizeof(v), cudaMemcpyHostToDevice, c->stream));
  const double z = 0.0;
  CK(cudaMemcpyAsync(c->d_scal + 7, &z, sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->d_scal + 9, &z, sizeof(double), cudaMemcpyHostToDevice, c->stream));  // it_init = it
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

int amrvac_gpu_step(amrvac_ctx *c) {
  if (int r = check_ctx(c, true)) return r;
  return launch_step(c);
}

int amrvac_gpu_run(amrvac_ctx *c, int nsteps) {
  if (int r = check_ctx(c, true)) return r;
  if (nsteps <= 0) return 0;
  if (!c->graph) {
    cudaGraph_t g;
    const int64_t before = c->launches;
    CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    int r = launch_step(c);
    cudaError_t e = cudaStreamEndCapture(c->stream, &g);
    if (r) { if (e == cudaSuccess) cudaGraphDestroy(g); return r; }
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
    c->graph_nodes = c->launches - before;
    c->launches = before;
    e = cudaGraphInstantiate(&c->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) { c->graph = nullptr; return cuda_fail(e, "cudaGraphInstantiate"); }
  }
  for (int s = 0; s < nsteps; ++s) {
    CK(cudaGraphLaunch(c->graph, c->stream));
    c->launches += c->graph_nodes;
  }
  return 0;
}

int amrvac_gpu_run_timed(amrvac_ctx *c, int nsteps, double *total_ms, double *stage_ms, double *getdt_ms) {
  if (int r = check_ctx(c, true)) return r;
  if (c->cfg.dimsplit) return fail(AMRVAC_E_UNSUPPORTED, "run_timed: dimsplit (use amrvac_gpu_step / run)");
  if (nsteps <= 0) return fail(AMRVAC_E_ARG, "nsteps must be positive");
  const int nst = c->cfg.time_stepper;  // stages per step
  const int per = 3 + nst;              // events per step
  std::vector<cudaEvent_t> ev((size_t)nsteps * per + 1);
  for (auto &e : ev) CK(cudaEventCreate(&e));
  int r = 0;
  size_t q = 0;
  CK(cudaEventRecord(ev[q++], c->stream));
  for (int s = 0; s < nsteps && !r; ++s) {
    r = launch_getdt(c, 0);
    if (r) break;
    CK(cudaEventRecord(ev[q++], c->stream));  // after getdt
    CK(launch_setdt_finalize(c->d_red, c->d_scal, c->d_status, c->stream));
    ++c->launches;
    CK(cudaEventRecord(ev[q++], c->stream));  // before stage 1
    const amrvac_cfg &k = c->cfg;
    if (k.time_stepper == AMRVAC_TS_ONESTEP) {
      CK(cudaMemcpyAsync(c->pool[1], c->pool[0], sizeof(double) * c->per_block * c->nw * c->nblocks,
                         cudaMemcpyDeviceToDevice, c->stream));
      r = launch_stage(c, 1, 0, 0, 0.0, 1.0, 1.0);
      CK(cudaEventRecord(ev[q++], c->stream));
    } else if (k.time_stepper == AMRVAC_TS_TWOSTEP) {
      const bool pc = k.time_integrator != AMRVAC_TI_SSPRK2;
      r = pc ? launch_stage(c, 0, 1, 0, 0.0, 1.0, 0.5, false, uses_hancock(k)) : launch_stage(c, 0, 1, 0, 0.0, 1.0, 1.0);
      CK(cudaEventRecord(ev[q++], c->stream));
      if (!r) r = pc ? launch_stage(c, 1, 0, 0, 1.0, 0.0, 1.0) : launch_stage(c, 1, 0, 0, 0.5, 0.5, 0.5);
      CK(cudaEventRecord(ev[q++], c->stream));
    } else if (k.time_stepper == AMRVAC_TS_FOURSTEP) {
      r = launch_fourstep(c, &ev[q]);
      q += 4;
    } else if (k.time_stepper == AMRVAC_TS_FIVESTEP) {
      r = launch_fivestep(c, &ev[q]);
      q += 5;
    } else {
      double b11, b22, b33, a21, a31;
      if (k.ssprk_order == 2) { b11 = 0.5; b22 = 0.5; b33 = 1.0 / 3.0; a21 = 0.0; a31 = 1.0 / 3.0; }
      else { b11 = 1.0; b22 = 1.0 / 4.0; b33 = 2.0 / 3.0; a21 = 3.0 / 4.0; a31 = 1.0 / 3.0; }
      r = launch_stage(c, 0, 1, 0, 0.0, 1.0, b11);
      CK(cudaEventRecord(ev[q++], c->stream));
      if (!r) r = launch_stage(c, 1, 2, 0, a21, 1.0 - a21, b22);
      CK(cudaEventRecord(ev[q++], c->stream));
      if (!r) r = launch_stage(c, 2, 0, 0, a31, 1.0 - a31, b33);
      CK(cudaEventRecord(ev[q++], c->stream));
    }
    CK(launch_advance_time(c->d_scal, c->stream));
    ++c->launches;
    CK(cudaEventRecord(ev[q++], c->stream));  // end of step
  }
  CK(cudaStreamSynchronize(c->stream));
  double tot = 0, st = 0, gd = 0;
  float ms;
  if (!r) {
    CK(cudaEventElapsedTime(&ms, ev[0], ev[q - 1]));
    tot = ms;
    size_t base = 1;
    cudaEvent_t prev_end = ev[0];
    for (int s = 0; s < nsteps; ++s) {
      CK(cudaEventElapsedTime(&ms, prev_end, ev[base]));  // getdt
      gd += ms;
      for (int k2 = 0; k2 < nst; ++k2) {
        CK(cudaEventElapsedTime(&ms, ev[base + 1 + k2], ev[base + 2 + k2]));
        st += ms;
      }
      prev_end = ev[base + 2 + nst];
      base += per;
    }
  }
  for (auto &e : ev) cudaEventDestroy(e);
  if (r) return r;
  if (total_ms) *total_ms = tot;
  if (stage_ms) *stage_ms = st;
  if (getdt_ms) *getdt_ms = gd;
  return 0;
}

int amrvac_gpu_set_zchunk(amrvac_ctx *c, int zchunk) {
  if (int r = check_ctx(c, false)) return r;
  if (!valid_zchunk(c->bn, zchunk))
    return fail(AMRVAC_E_ARG, "zchunk must be 0 (persistent plane ranges) or a divisor >= 2 of block_nx");
  if (c->graph) { cudaGraphExecDestroy(c->graph); c->graph = nullptr; }
  c->zchunk = zchunk;
  return 0;
}

int amrvac_gpu_set_stage_variant(amrvac_ctx *c, int var) {
  if (int r = check_ctx(c, false)) return r;
  if (var < 0 || var >= c->ks.nvar) return fail(AMRVAC_E_ARG, "no such stage-kernel variant for this scheme");
  if (c->graph) { cudaGraphExecDestroy(c->graph); c->graph = nullptr; }
  c->var = var;
  return 0;
}

int amrvac_gpu_stage_variant(amrvac_ctx *c, int *var, int *nvar, int *threads, int *ctas_per_sm, int *async) {
  if (int r = check_ctx(c, false)) return r;
  if (var) *var = c->var;
  if (nvar) *nvar = c->ks.nvar;
  if (threads) *threads = c->ks.var_threads[c->var];
  if (ctas_per_sm) *ctas_per_sm = c->ks.var_minb[c->var];
  if (async) *async = c->ks.var_async[c->var];
  return 0;
}

int amrvac_gpu_autotune(amrvac_ctx *c, int reps, int *best_zchunk, double *best_ms) {
  if (int r = check_ctx(c, true)) return r;
  if (reps <= 0) reps = 3;
  // persistent, then z-chunks of the whole block, a half and a quarter of it
  const int bn = c->bn;
  int cand[4] = {0, bn, 0, 0}, ncand = 2;
  if (c->cfg.ndim == 3) {
    if (valid_zchunk(bn, bn / 2) && bn % 2 == 0) cand[ncand++] = bn / 2;
    if (bn % 4 == 0 && valid_zchunk(bn, bn / 4)) cand[ncand++] = bn / 4;
  }
  // dt and cmax_global of the current state (GLM needs cmax_global > 0)
  if (int r = launch_getdt(c, 0)) return r;
  CK(launch_setdt_finalize(c->d_red, c->d_scal, c->d_status, c->stream));
  ++c->launches;
  cudaEvent_t a, b;
  CK(cudaEventCreate(&a));
  CK(cudaEventCreate(&b));
  // every stage-kernel variant of the scheme with every work distribution
  int best = c->zchunk, bvar = c->var;
  float bms = 1e30f;
  for (int v = 0; v < c->ks.nvar; ++v) {
    c->var = v;
    for (int q = 0; q < ncand; ++q) {
      c->zchunk = cand[q];
      int r = launch_stage(c, 0, 1, 0, 0.0, 1.0, 1.0);  // warm
      CK(cudaEventRecord(a, c->stream));
      for (int i = 0; i < reps && !r; ++i) r = launch_stage(c, 0, 1, 0, 0.0, 1.0, 1.0);
      CK(cudaEventRecord(b, c->stream));
      CK(cudaEventSynchronize(b));
      if (r) { cudaEventDestroy(a); cudaEventDestroy(b); return r; }
      float ms;
      CK(cudaEventElapsedTime(&ms, a, b));
      ms /= reps;
      if (ms < bms) { bms = ms; best = cand[q]; bvar = v; }
    }
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  c->zchunk = best;
  c->var = bvar;
  if (c->graph) { cudaGraphExecDestroy(c->graph); c->graph = nullptr; }
  if (best_zchunk) *best_zchunk = best;
  if (best_ms) *best_ms = bms;
  return 0;
}

int amrvac_gpu_wait_probe(int spins, uint32_t *flags) {
  if (!flags || spins < 1 || spins > AMRVAC_ASYNC_SPINS) return fail(AMRVAC_E_ARG, "wait_probe: bad arguments");
  if (cudaError_t e = run_wait_probe(spins, flags)) return cuda_fail(e, "wait_probe");
  return 0;
}

int amrvac_gpu_fp64_peak(double *tflops) {
  if (!tflops) return fail(AMRVAC_E_ARG, "null pointer");
  CK(measure_fp64_peak(tflops));
  return 0;
}

int amrvac_gpu_get_time(amrvac_ctx *c, double *dt, double *cmax_global, double *global_time) {
  if (int r = check_ctx(c, false)) return r;
  double s[3];
  CK(cudaMemcpyAsync(s, c->d_scal, sizeof(s), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (dt) *dt = s[0];
  if (cmax_global) *cmax_global = s[1];
  if (global_time) *global_time = s[2];
  return 0;
}

int amrvac_gpu_status(amrvac_ctx *c, uint32_t *flags) {
  if (int r = check_ctx(c, false)) return r;
  if (!flags) return fail(AMRVAC_E_ARG, "null flags");
  CK(cudaMemcpyAsync(flags, c->d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

int amrvac_gpu_clear_status(amrvac_ctx *c) {
  if (int r = check_ctx(c, false)) return r;
  CK(cudaMemsetAsync(c->d_status, 0, sizeof(uint32_t), c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

int amrvac_gpu_synchronize(amrvac_ctx *c) {
  if (int r = check_ctx(c, false)) return r;
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

int amrvac_gpu_stream(amrvac_ctx *c, void **stream) {
  if (int r = check_ctx(c, false)) return r;
  if (!stream) return fail(AMRVAC_E_ARG, "null stream pointer");
  *stream = (void *)c->stream;
  return 0;
}

int amrvac_gpu_register_ptr(amrvac_ctx *c, int reg, double **dptr) {
  if (int r = check_ctx(c, true)) return r;
  if (reg < 0 || reg > 2 || !dptr) return fail(AMRVAC_E_ARG, "bad register");
  *dptr = c->pool[reg];
  return 0;
}

int64_t amrvac_gpu_launch_count(const amrvac_ctx *c) { return c ? c->launches : -1; }

// ---------------------------------------------------------------- points
static int run_points(amrvac_ctx *c, int n, int idim, const double *a, const double *b, const double *cc,
                      const double *d, double *out, size_t out_per, double *out2, double cg, int kind) {
  if (int r = check_ctx(c, false)) return r;
  if (n <= 0 || !a || !out) return fail(AMRVAC_E_ARG, "bad points arguments");
  const size_t sz = (size_t)n * c->nw;
  double *dev = nullptr;
  const size_t total = sz * 4 + (size_t)n * out_per + (size_t)n;
  CK(cudaMalloc(&dev, sizeof(double) * total));
  double *da = dev, *db = dev + sz, *dc = dev + 2 * sz, *dd = dev + 3 * sz, *dout = dev + 4 * sz,
         *dout2 = dout + (size_t)n * out_per;
  auto up = [&](double *dst, const double *src) -> cudaError_t {
    return src ? cudaMemcpyAsync(dst, src, sizeof(double) * sz, cudaMemcpyHostToDevice, c->stream) : cudaSuccess;
  };
  PointArgs A;
  A.n = n; A.a = da; A.b = db; A.c = dc; A.d = dd; A.out = dout; A.out2 = out2 ? dout2 : nullptr;
  A.cg = cg; A.P = c->P;
  cudaError_t e = up(da, a);
  if (e == cudaSuccess) e = up(db, b);
  if (e == cudaSuccess) e = up(dc, cc);
  if (e == cudaSuccess) e = up(dd, d);
  if (e == cudaSuccess) {
    if (kind == 0) e = c->ks.riemann_points(A, idim, c->stream);
    else if (kind == 1) e = c->ks.flux_points(A, idim, c->stream);
    else e = c->ks.cbounds_points(A, idim, c->stream);
    ++c->launches;
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(out, dout, sizeof(double) * n * out_per, cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess && out2) e = cudaMemcpyAsync(out2, dout2, sizeof(double) * n, cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  cudaFree(dev);
  if (e != cudaSuccess) return cuda_fail(e, "points kernel");
  return 0;
}

int amrvac_gpu_riemann_points(amrvac_ctx *c, int n, const double *wlp, const double *wrp, int idim,
                              double cmax_global, double *f) {
  if (!c) return fail(AMRVAC_E_ARG, "null context");
  if (idim < 1 || idim > c->cfg.ndim) return fail(AMRVAC_E_ARG, "idim out of range");
  return run_points(c, n, idim, wlp, wrp, nullptr, nullptr, f, c->nw, nullptr, cmax_global, 0);
}

int amrvac_gpu_get_flux_points(amrvac_ctx *c, int n, const double *wc, const double *wp, int idim,
                               double cmax_global, double *f) {
  if (!c) return fail(AMRVAC_E_ARG, "null context");
  if (idim < 1 || idim > c->cfg.ndir) return fail(AMRVAC_E_ARG, "idim out of range");
  return run_points(c, n, idim, wc, wp, nullptr, nullptr, f, c->nw, nullptr, cmax_global, 1);
}

int amrvac_gpu_get_cbounds_points(amrvac_ctx *c, int n, const double *wlc, const double *wrc,
                                  const double *wlp, const double *wrp, int idim, double *cmax,
                                  double *cmin) {
  if (!c) return fail(AMRVAC_E_ARG, "null context");
  if (idim < 1 || idim > c->cfg.ndir) return fail(AMRVAC_E_ARG, "idim out of range");
  return run_points(c, n, idim, wlc, wrc, wlp, wrp, cmax, 1, cmin, 0.0, 2);
}

int amrvac_gpu_div_points(int n, const double *x, const double *y, double *q, double *r, double *seed) {
  if (n <= 0 || !x || !y || !q || !r || !seed) return fail(AMRVAC_E_ARG, "div_points: bad arguments");
  const size_t b = sizeof(double) * (size_t)n;
  double *d = nullptr;
  CK(cudaMalloc(&d, 5 * b));
  cudaError_t e = cudaMemcpy(d, x, b, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d + n, y, b, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = launch_div_points(n, d, d + n, d + 2 * (size_t)n, d + 3 * (size_t)n, d + 4 * (size_t)n, 0);
  if (e == cudaSuccess) e = cudaMemcpy(q, d + 2 * (size_t)n, b, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(r, d + 3 * (size_t)n, b, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(seed, d + 4 * (size_t)n, b, cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) return cuda_fail(e, "div_points");
  return 0;
}


// ---------------------------------------------------------------- adjoint
int amrvac_gpu_step_dt(amrvac_ctx *c, double dt) {
  if (int r = check_ctx(c, true)) return r;
  if (!(dt > 0.0)) return fail(AMRVAC_E_ARG, "dt must be positive");
  if (int r = check_a2max(c)) return r;
  CK(launch_set_scalar(c->d_scal + 0, dt, c->stream));
  ++c->launches;
  return launch_rk(c);
}

int amrvac_gpu_register_copy(amrvac_ctx *c, int reg, double *dev, int to_register) {
  if (int r = check_ctx(c, true)) return r;
  if (reg < 0 || reg > 2 || !dev) return fail(AMRVAC_E_ARG, "bad register copy");
  const size_t bytes = sizeof(double) * c->per_block * c->nw * c->nblocks;
  CK(cudaMemcpyAsync(to_register ? c->pool[reg] : dev, to_register ? dev : c->pool[reg], bytes,
                     cudaMemcpyDeviceToDevice, c->stream));
  return 0;
}

// One step at dt whose stage inputs and result live in the caller's buffers.
// The stages are those of launch_rk (same kernels, coefficients and order),
// with the registers pointed at the caller's buffers for the duration of the
// call: stage 1 reads u0 and writes u1, stage 2 writes u2 (threestep), the
// last stage writes unew (which may be u0: its base is read cell by cell).
int amrvac_gpu_step_dt_states(amrvac_ctx *c, double dt, const double *u0, double *u1, double *u2, double *unew) {
  if (int r = check_ctx(c, true)) return r;
  const amrvac_cfg &k = c->cfg;
  const bool three = k.time_stepper == AMRVAC_TS_THREESTEP;
  if (!three && !(k.time_stepper == AMRVAC_TS_TWOSTEP && k.time_integrator == AMRVAC_TI_SSPRK2))
    return fail(AMRVAC_E_UNSUPPORTED, "step_dt_states: threestep or twostep with time_integrator ssprk2");
  if (c->amr || k.dimsplit || c->sv_on)
    return fail(AMRVAC_E_UNSUPPORTED, "step_dt_states: single-level unsplit grids, no small_values average");
  if (!(dt > 0.0)) return fail(AMRVAC_E_ARG, "dt must be positive");
  if (!u0 || !u1 || (three && !u2)) return fail(AMRVAC_E_ARG, "step_dt_states: null stage buffer");
  // distinct stage inputs; U^{n+1} may replace u0 only (a stage reads its
  // input's neighbours, its base cell by cell)
  if (u1 == u0 || (three && (u2 == u0 || u2 == u1)))
    return fail(AMRVAC_E_ARG, "step_dt_states: u0, u1 and u2 must be distinct buffers");
  if (unew && (unew == u1 || (three && unew == u2)))
    return fail(AMRVAC_E_ARG, "step_dt_states: unew must be u0 or a buffer of its own");
  if (int r = check_a2max(c)) return r;
  CK(launch_set_scalar(c->d_scal + 0, dt, c->stream));
  ++c->launches;
  double *const saved[3] = {c->pool[0], c->pool[1], c->pool[2]};
  c->pool[0] = const_cast<double *>(u0);  // read only: every stage takes it as input or base
  c->pool[1] = u1;
  int r;
  if (!three) {
    r = launch_stage(c, 0, 1, 0, 0.0, 1.0, 1.0);
    if (!r && unew) {
      c->pool[2] = unew;
      r = launch_stage(c, 1, 2, 0, 0.5, 0.5, 0.5);
    }
  } else {
    double b11, b22, b33, a21, a31;
    if (k.ssprk_order == 2) { b11 = 0.5; b22 = 0.5; b33 = 1.0 / 3.0; a21 = 0.0; a31 = 1.0 / 3.0; }
    else { b11 = 1.0; b22 = 1.0 / 4.0; b33 = 2.0 / 3.0; a21 = 3.0 / 4.0; a31 = 1.0 / 3.0; }
    c->pool[2] = u2;
    r = launch_stage(c, 0, 1, 0, 0.0, 1.0, b11);
    if (!r) r = launch_stage(c, 1, 2, 0, a21, 1.0 - a21, b22);
    if (!r && unew) {
      c->pool[1] = unew;
      r = launch_stage(c, 2, 1, 0, a31, 1.0 - a31, b33);
    }
  }
  for (int i = 0; i < 3; ++i) c->pool[i] = saved[i];
  return r;
}

static int adjoint_step_impl(amrvac_ctx *c, const double *u0, const double *u1, const double *u2, double *lam,
                             double dt, double *gamma_part);

int amrvac_gpu_adjoint_step(amrvac_ctx *c, double *lam, double dt, double *gamma_part) {
  return adjoint_step_impl(c, nullptr, nullptr, nullptr, lam, dt, gamma_part);
}

int amrvac_gpu_adjoint_step_states(amrvac_ctx *c, const double *u0, const double *u1, const double *u2, double *lam,
                                   double dt, double *gamma_part) {
  if (!u0 || !u1 || (!u2 && c && c->cfg.time_stepper == AMRVAC_TS_THREESTEP))
    return fail(AMRVAC_E_ARG, "adjoint_step_states: null stage state");
  return adjoint_step_impl(c, u0, u1, u2, lam, dt, gamma_part);
}

static int adjoint_step_impl(amrvac_ctx *c, const double *u0, const double *u1, const double *u2, double *lam,
                             double dt, double *gamma_part) {
  if (int r = check_ctx(c, true)) return r;
  const amrvac_cfg &k = c->cfg;
  if (!lam || !gamma_part || !(dt > 0.0)) return fail(AMRVAC_E_ARG, "bad adjoint arguments");
  if (c->amr) return fail(AMRVAC_E_UNSUPPORTED, "adjoint: single-level grids only");
  if (c->sv_on) return fail(AMRVAC_E_UNSUPPORTED, "adjoint: not with small_values_method average");
  if (k.physics != 0 || k.ndim != 2 || (k.flux_scheme != AMRVAC_FS_HLL && k.flux_scheme != AMRVAC_FS_HLLC) ||
      k.typeboundspeed != AMRVAC_BS_EINFELDT || (k.limiter != AMRVAC_LIM_MINMOD && k.limiter != AMRVAC_LIM_VANLEER) ||
      k.fix_small_values || k.precision != 0)
    return fail(AMRVAC_E_UNSUPPORTED,
                "adjoint: 2-D hd, hll or hllc, minmod or vanleer, Einfeldt, FP64, no fix_small_values");
  if (k.time_stepper != AMRVAC_TS_THREESTEP &&
      !(k.time_stepper == AMRVAC_TS_TWOSTEP && k.time_integrator == AMRVAC_TI_SSPRK2))
    return fail(AMRVAC_E_UNSUPPORTED, "adjoint: threestep or twostep with time_integrator ssprk2");
  for (int sd = 0; sd < 4; ++sd)
    if (c->bc.kind[sd] == BCK_MIRROR) return fail(AMRVAC_E_UNSUPPORTED, "adjoint: periodic or cont boundaries");
  for (int b = 1; b < c->nblocks; ++b)
    for (int d = 0; d < 2; ++d)
      if (c->h_dx[(size_t)b * 3 + d] != c->h_dx[d]) return fail(AMRVAC_E_UNSUPPORTED, "adjoint: uniform dx");
  if (!c->adj_prepared) {
    CK(adjoint_prepare());
    c->adj_prepared = true;
  }
  const size_t bytes = sizeof(double) * c->per_block * c->nw * c->nblocks;
  for (int r = 0; r < 3; ++r)
    if (!c->d_adj[r]) CK(cudaMalloc(&c->d_adj[r], bytes));
  double *S1 = c->d_adj[0], *S2 = c->d_adj[1], *S3 = c->d_adj[2];
  // stage inputs: the caller's buffers, or registers 0..2 recomputed below
  const double *W[3] = {u0 ? u0 : c->pool[0], u1 ? u1 : c->pool[1], u2 ? u2 : c->pool[2]};
  auto args = [&](int reg_w, const double *lam_new, double *out, const double *acc, double *base, int binit,
                  double a, double b, double dtf) {
    AdjArgs A;
    std::memset(&A, 0, sizeof(A));
    A.sa = stage_args(c, reg_w, reg_w, reg_w, 0.0, 1.0, 1.0);
    A.sa.uin = W[reg_w];
    A.lam = lam_new;
    A.lam_out = out;
    A.acc_in = acc;
    A.base = base;
    A.base_init = binit;
    A.a = a;
    A.b = b;
    for (int d = 0; d < 2; ++d) A.s[d] = dtf * dt / c->h_dx[d];
    A.gamma_part = gamma_part;
    return A;
  };
  CK(launch_set_scalar(c->d_scal + 0, dt, c->stream));
  ++c->launches;
  if (k.time_stepper == AMRVAC_TS_TWOSTEP) {
    // forward U1 = U0 + dt L(U0); U2 = (U0 + U1 + dt L(U1)) / 2
    if (!u0)
      if (int r = launch_stage(c, 0, 1, 0, 0.0, 1.0, 1.0)) return r;
    CK(launch_adjoint_stage(args(1, lam, S1, nullptr, S2, 1, 0.5, 0.5, 0.5), k.limiter, k.flux_scheme, c->stream));
    CK(launch_adjoint_stage(args(0, S1, lam, S2, nullptr, 0, 0.0, 1.0, 1.0), k.limiter, k.flux_scheme, c->stream));
    c->launches += 3;
    return 0;
  }
  double b11, b22, b33, a21, a31;
  if (k.ssprk_order == 2) { b11 = 0.5; b22 = 0.5; b33 = 1.0 / 3.0; a21 = 0.0; a31 = 1.0 / 3.0; }
  else { b11 = 1.0; b22 = 1.0 / 4.0; b33 = 2.0 / 3.0; a21 = 3.0 / 4.0; a31 = 1.0 / 3.0; }
  // recompute the stage inputs U1 (register 1) and U2 (register 2) from U^n (register 0)
  if (!u0) {
    if (int r = launch_stage(c, 0, 1, 0, 0.0, 1.0, b11)) return r;
    if (int r = launch_stage(c, 1, 2, 0, a21, 1.0 - a21, b22)) return r;
  }
  // stage 3: U3 = a31 U0 + (1-a31) U2 + b33 dt L(U2)
  CK(launch_adjoint_stage(args(2, lam, S1, nullptr, S2, 1, a31, 1.0 - a31, b33), k.limiter, k.flux_scheme, c->stream));
  // stage 2: U2 = a21 U0 + (1-a21) U1 + b22 dt L(U1)
  CK(launch_adjoint_stage(args(1, S1, S3, nullptr, S2, 0, a21, 1.0 - a21, b22), k.limiter, k.flux_scheme, c->stream));
  // stage 1: U1 = U0 + b11 dt L(U0); dL/dU0 = base sum + stage-1 transpose
  CK(launch_adjoint_stage(args(0, S3, lam, S2, nullptr, 0, 0.0, 1.0, b11), k.limiter, k.flux_scheme, c->stream));
  c->launches += 3;
  return 0;
}


// ---------------------------------------------------------------- AMR decisions
int amrvac_gpu_lohner(amrvac_ctx *c, int reg, const double *weight, const int *logflag, int refine_max_level,
                      const double *refine_threshold, const double *derefine_ratio, const double *amr_wavefilter,
                      const int *block_level, int *flags, double *errmax) {
  if (int r = check_ctx(c, true)) return r;
  if (reg < 0 || reg > 2 || !weight || !flags || !refine_threshold || !derefine_ratio || !amr_wavefilter)
    return fail(AMRVAC_E_ARG, "lohner: bad arguments");
  if (refine_max_level < 1 || refine_max_level > AMR_MAX_LEVELS)
    return fail(AMRVAC_E_ARG, "lohner: refine_max_level out of range");
  if (c->cfg.ndim < 2) return fail(AMRVAC_E_UNSUPPORTED, "lohner: ndim 2 or 3");
  LohnerArgs A;
  std::memset(&A, 0, sizeof(A));
  if (c->amr)
    if (int r = launch_amr_ghost_pass(c, reg)) return r;
  A.sa = stage_args(c, reg, reg, reg, 0.0, 1.0, 1.0);
  A.nw = c->nw;
  for (int v = 0; v < c->nw; ++v) {
    A.weight[v] = weight[v];
    if (logflag && logflag[v]) A.logflag |= 1u << v;
  }
  for (int l = 0; l < refine_max_level; ++l) {
    A.threshold[l] = refine_threshold[l];
    A.derefine[l] = derefine_ratio[l];
    A.wavefilter[l] = amr_wavefilter[l];
  }
  A.refine_max_level = refine_max_level;
  std::vector<int> lev(c->nblocks, 1);
  if (block_level)
    for (int b = 0; b < c->nblocks; ++b) {
      if (block_level[b] < 1 || block_level[b] > refine_max_level) return fail(AMRVAC_E_ARG, "lohner: bad level");
      lev[b] = block_level[b];
    }
  if ((size_t)c->nblocks > c->amr_int_cap || !c->d_amr_int) {
    cudaFree(c->d_amr_int);
    cudaFree(c->d_amr_err);
    c->d_amr_int = nullptr;
    c->d_amr_err = nullptr;
    c->amr_int_cap = 0;
    const size_t cap = (size_t)c->nblocks + c->nblocks / 4 + 1;
    CK(cudaMalloc(&c->d_amr_int, sizeof(int) * 2 * cap));
    CK(cudaMalloc(&c->d_amr_err, sizeof(double) * cap));
    c->amr_int_cap = cap;
  }
  CK(cudaMemcpyAsync(c->d_amr_int, lev.data(), sizeof(int) * c->nblocks, cudaMemcpyHostToDevice, c->stream));
  A.level = c->d_amr_int;
  A.flags = c->d_amr_int + c->nblocks;
  A.errmax = c->d_amr_err;
  CK(launch_lohner(A, c->cfg.ndim, c->stream));
  ++c->launches;
  CK(cudaMemcpyAsync(flags, A.flags, sizeof(int) * c->nblocks, cudaMemcpyDeviceToHost, c->stream));
  if (errmax) CK(cudaMemcpyAsync(errmax, c->d_amr_err, sizeof(double) * c->nblocks, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

}  // extern "C"
