// Fused finite-volume stage kernel for 16^d blocks (d = 2, 3).
//
// One CTA advances one block (or a z-chunk of a 3-D block) by one explicit
// stage.  It restates, for all cells of its tile at once:
//   finite_volume (src/mod_finite_volume.t:116-339): primitives, limited
//     reconstruction (reconstruct_LR 1110-1228), GLM modify_wLR, physical
//     fluxes, signal-speed bounds, Riemann flux, conservative update;
//   the SSP-RK stage combination (src/mod_advance.t:249-267);
//   the divB sources (add_source_glm / add_source_linde,
//     src/mhd/mod_mhd_phys.t:5472-5531, 5599-5665);
//   the same-resolution ghost fill (bc_fill_srl, src/mod_ghostcells_update.t:
//     812-852) and cont/symm/asymm physical boundaries, done as a gather from
//     the neighbour blocks' interiors while staging the tile.
//
// Layout in HBM: pool[block][var][z][y][x], interior cells only, 16^d per
// block and variable (2 KB rows of 16 doubles).  No ghost cells are stored.
//
// CTA organisation (3-D): 256 threads march over the z-planes of the tile.
// Shared memory holds a ring of 2 HW primitive planes (HW = 2 halo cells,
// 3 for the fifth-order reconstructions; planes k-HW+1 .. k+HW, 16x16 each),
// the x/y halo strips of plane k, one buffer of scaled face fluxes and a
// 16-face side buffer.  Per plane: the 17x16 x-faces together with the 16
// y-faces of the top row (288 faces: a second round of one warp), per-cell
// accumulation, the remaining 16x16 y-faces, accumulation, then each cell
// thread computes its own z-face k+1/2 and keeps the k-1/2 flux in
// registers.  Variants of the same kernel: the MUSCL-Hancock predictor
// (per-cell edge fluxes, no Riemann solver) and dimensionally split sweeps
// (one direction per launch).
#pragma once

#include <cuda_runtime.h>

#include "physics.cuh"
#include "riemann.cuh"

namespace amrvac {

// Block edge (block_nx, the same in every direction).  The reference allows
// any even block_nx >= 4 (src/io/mod_input_output.t:1494-1503); the library
// runs the sizes of BLOCK_SIZES.  Helpers that address blocks take the edge
// as an argument (a constant in the stage kernel, so it folds there).
constexpr int BN16 = 16;
// The stage kernel advances a tile of TB x TB cells of a block's z-plane per
// CTA: the whole plane up to block_nx 16, else the largest divisor of
// block_nx that is at most 16 (32 -> four 16 x 16 tiles per plane).
__host__ __device__ constexpr int tile_edge(int bn) {
  if (bn <= 16) return bn;
  for (int t = 16; t > 1; --t)
    if (bn % t == 0) return t;
  return 1;
}
// The block edges the library's kernels are built for.
__host__ __device__ constexpr bool block_edge_built(int bn) {
  return bn == 8 || bn == 10 || bn == 12 || bn == 16 || bn == 32;
}
// threads of a stage CTA: one per cell of the tile, rounded up to whole warps
__host__ __device__ constexpr int stage_threads(int bn) {
  return (tile_edge(bn) * tile_edge(bn) + 31) / 32 * 32;
}
#ifndef AMRVAC_STAGE_THREADS
#define AMRVAC_STAGE_THREADS 256
#endif
#ifndef AMRVAC_STAGE_MINB
#define AMRVAC_STAGE_MINB 2
#endif
#ifndef AMRVAC_STAGE_MINB_MIXED
#define AMRVAC_STAGE_MINB_MIXED 3
#endif
// 256 threads x 2 CTAs per SM (128 registers per thread, shared memory
// 104 KB per CTA for nw = 9): the two CTAs hide each other's barrier and
// dependency stalls; the 16 extra faces of an x/y phase (17x16 faces per
// plane) take a second, partial round.  (288 threads x 1 CTA, one face per
// thread, measured 17-25 % slower on 3-D MHD.)
constexpr int STAGE_THREADS = AMRVAC_STAGE_THREADS;

enum : int { BCK_PERIODIC = 0, BCK_CONT = 1, BCK_MIRROR = 2 };

struct StageArgs {
  const double *uin;        // register holding wCT
  const double *ubase;      // register holding the RK base (may alias uout)
  double *uout;             // register receiving wnew
  double a_base, b_in;      // wnew0 = a_base*base + b_in*in (a_base==0: wnew0 = in)
  double dtfactor;
  const double *dt_dev;     // device scalar dt
  const double *cmax_dev;   // device scalar cmax_global (GLM)
  const int *nbr;           // [nblocks][27] neighbour block or -1 (physical boundary)
  const double *dxb;        // [nblocks][3] cell size per block
  int nblocks;
  int zchunk;               // z-planes per CTA (3-D); 16 = whole block
  int bc_kind[6];           // per side: BCK_*
  uint32_t bc_flip[6];      // per side: bit v set -> variable v changes sign (asymm)
  uint32_t *status;         // global status word (atomicOr)
  uint32_t *block_status;   // [nblocks] per-block status (crash restore)
  PhysParams P;
  // Multi-level grids (all null on a single level).  A neighbour entry
  // <= -2 means "the ghost cells of this direction are in the block's ghost
  // buffer gbuf[-2 - entry]" (restricted or prolonged values, written by the
  // AMR ghost pass); amr_face[b] bit 2d+side marks a level jump across that
  // face, whose boundary face fluxes are stored in pflux[gslot[b]].
  const double *gbuf;       // [slot][var][gz][gy][gx], ghosted (2 layers)
  double *pflux;            // [slot][2*ndim][var][16*16] scaled face fluxes
  const int *gslot;         // [nblocks] slot or -1
  const int *amr_face;      // [nblocks] bitmask
  // Dimensional splitting: sweep < 0 advances all directions; otherwise the
  // stage is the sweep-th of the step's one-direction sweeps (see sweep_dir).
  int sweep;
  int split_xy;             // 1: typedimsplit 'xy' (same order every step)
  int bn;                   // block edge, for the kernels that take it at run time
};

// Direction of a dimensionally split sweep (src/mod_advance.t:23-45):
// increasing order on even steps (and always with typedimsplit 'xy'),
// decreasing on odd steps ('xyyx'); the step count is the device scalar
// scal[9] (steps since set_time).  -1: unsplit.
__device__ __forceinline__ int sweep_dir(int sweep, int split_xy, const double *scal, int ndim) {
  if (sweep < 0) return -1;
  const long it = (long)scal[9];
  return (split_xy || (it & 1L) == 0) ? sweep : ndim - 1 - sweep;
}

__device__ __forceinline__ int dir_index(int di, int dj, int dk) {
  return (di + 1) + 3 * (dj + 1) + 9 * (dk + 1);
}

// Resolve a cell of block b (edge bn) given local coordinates that may lie
// up to two (three with MP5) cells outside the block: physical sides first
// (clamp for cont, mirror for symm/asymm), then the remaining offset through
// the neighbour table.
template <int NDIM>
__device__ __forceinline__ int resolve_cell(const StageArgs &A, int b, int &i, int &j, int &k,
                                            uint32_t &flip, int BN = BN16) {
  int c[3] = {i, j, k};
  int dir[3] = {0, 0, 0};
  flip = 0;
#pragma unroll
  for (int d = 0; d < NDIM; ++d) {
    int side = c[d] < 0 ? 0 : (c[d] >= BN ? 1 : -1);
    if (side < 0) continue;
    int fd[3] = {0, 0, 0};
    fd[d] = side ? 1 : -1;
    const int nf = A.nbr[b * 27 + dir_index(fd[0], fd[1], fd[2])];
    if (nf == -1) {
      const int kind = A.bc_kind[2 * d + side];
      if (kind == BCK_CONT) {
        c[d] = side ? BN - 1 : 0;
      } else {
        c[d] = side ? 2 * BN - 1 - c[d] : -1 - c[d];
        flip ^= A.bc_flip[2 * d + side];
      }
    } else {
      dir[d] = side ? 1 : -1;
    }
  }
  int blk = b;
  if (dir[0] | dir[1] | dir[2]) {
    blk = A.nbr[b * 27 + dir_index(dir[0], dir[1], dir[2])];
    if (blk >= 0) {
#pragma unroll
      for (int d = 0; d < NDIM; ++d) c[d] -= dir[d] * BN;
    } else if (blk <= -2 && A.gbuf) {
      // level jump: the value is in this block's ghost buffer at c
    } else {  // inconsistent neighbour table: stay in bounds and flag it
      blk = b;
#pragma unroll
      for (int d = 0; d < NDIM; ++d) c[d] = min(max(c[d], 0), BN - 1);
      atomicOr(A.status, ST_BOUNDS);
    }
  }
  i = c[0]; j = c[1]; k = c[2];
  return blk;
}

template <int NDIM>
__device__ __forceinline__ size_t cell_offset(int blk, int nw, int v, int i, int j, int k, int BN = BN16) {
  const int NY = NDIM >= 2 ? BN : 1;
  const int NZ = NDIM >= 3 ? BN : 1;
  return (((size_t)blk * nw + v) * NZ + k) * (size_t)(NY * BN) + (size_t)j * BN + i;
}

// Offset of cell (i, j, k) (block-local, up to 2 outside) in a ghosted
// buffer of 2 ghost layers: [slot][var][gz][gy][gx].
template <int NDIM>
__device__ __forceinline__ size_t ghost_offset(int slot, int nw, int v, int i, int j, int k, int BN = BN16) {
  const int G = BN + 4;
  const int GY = NDIM >= 2 ? G : 1;
  const int GZ = NDIM >= 3 ? G : 1;
  const int gj = NDIM >= 2 ? j + 2 : 0, gk = NDIM >= 3 ? k + 2 : 0;
  return (((size_t)slot * nw + v) * GZ + gk) * (size_t)(GY * G) + (size_t)gj * G + (i + 2);
}

// Load the conserved state of a (possibly out-of-block) cell and return it
// as primitives.  Returns a status bit if the small-value check fires.
template <bool MHD, int NDIR, bool GLM, int NDIM, int BN = BN16>
__device__ __forceinline__ uint32_t load_prim(const StageArgs &A, int b, int i, int j, int k,
                                              double *w) {
  using V = Vars<MHD, NDIR, GLM>;
  uint32_t flip;
  const int blk = resolve_cell<NDIM>(A, b, i, j, k, flip, BN);
  if (blk >= 0) {
#pragma unroll
    for (int v = 0; v < V::NW; ++v) {
      double x = __ldg(A.uin + cell_offset<NDIM>(blk, V::NW, v, i, j, k, BN));
      w[v] = ((flip >> v) & 1u) ? -x : x;
    }
  } else {  // level jump: this block's ghost buffer
#pragma unroll
    for (int v = 0; v < V::NW; ++v) {
      const double x = __ldg(A.gbuf + ghost_offset<NDIM>(-2 - blk, V::NW, v, i, j, k, BN));
      w[v] = ((flip >> v) & 1u) ? -x : x;
    }
  }
  uint32_t st = 0;
  if (A.P.fix_small_values) {
    if (small_values<double, MHD, NDIR, GLM>(w, false, A.P) && A.P.small_values_method != 1) st |= ST_SMALL_VALUE;
  }
  to_primitive<MHD, NDIR, GLM>(w, A.P);
  return st;
}

// Interface flux from reconstructed primitive left/right states: small-value
// fix, to_conserved, GLM modify_wLR, physical fluxes, cbounds, Riemann solver
// (src/mod_finite_volume.t:1217-1222, 200-245).  wLp/wRp are modified.
template <class T, bool MHD, int NDIR, bool GLM, int NDIM, int SOLVER, int BS, bool FAST = false>
__device__ __forceinline__ uint32_t face_from_states(T *wLp, T *wRp, const PhysParams &P, T cg, T *F,
                                                     bool small_check = true) {
  constexpr int D = 0;  // states arrive rotated: the face normal is component 0
  using V = Vars<MHD, NDIR, GLM>;
  constexpr int NW = V::NW;
  uint32_t st = 0;
  if (small_check && P.fix_small_values) {
    bool fl = small_values<T, MHD, NDIR, GLM>(wLp, true, P);
    bool fr = small_values<T, MHD, NDIR, GLM>(wRp, true, P);
    if ((fl || fr) && P.small_values_method != 1) st |= ST_SMALL_VALUE;
  }
  T wLC[NW], wRC[NW];
#pragma unroll
  for (int v = 0; v < NW; ++v) { wLC[v] = wLp[v]; wRC[v] = wRp[v]; }
  to_conserved<T, MHD, NDIR, GLM>(wLC, P);
  to_conserved<T, MHD, NDIR, GLM>(wRC, P);
  if constexpr (MHD && GLM) {
    // mhd_modify_wLR (src/mhd/mod_mhd_phys.t:6352-6372)
    constexpr int BNI = V::B0 + D, PS = V::PSI, E = V::E;
    const T dB = wRp[BNI] - wLp[BNI];
    const T dPsi = wRp[PS] - wLp[PS];
    const T nb = T(0.5) * (wRp[BNI] + wLp[BNI] - div_f<FAST>(dPsi, cg));
    const T np = T(0.5) * (wRp[PS] + wLp[PS] - dB * cg);
    wLp[BNI] = nb; wLp[PS] = np; wRp[BNI] = nb; wRp[PS] = np;
    wRC[E] = wRC[E] - T(0.5) * (wRC[BNI] * wRC[BNI]);
    wLC[E] = wLC[E] - T(0.5) * (wLC[BNI] * wLC[BNI]);
    wRC[BNI] = nb; wRC[PS] = np; wLC[BNI] = nb; wLC[PS] = np;
    wRC[E] = wRC[E] + T(0.5) * (nb * nb);
    wLC[E] = wLC[E] + T(0.5) * (nb * nb);
  }
  T fL[NW], fR[NW];
  phys_flux<T, MHD, NDIR, GLM, D>(wLC, wLp, cg, fL);
  phys_flux<T, MHD, NDIR, GLM, D>(wRC, wRp, cg, fR);
  T cmax, cmin = T(0.0);
  if constexpr (SOLVER == SOLVER_TVDMU) {
    (void)cmax;
    if constexpr (MHD) {
      static_assert(!GLM, "TVD-MUSCL with GLM is not built");
      riemann_tvdmu_mhd<T, NDIR>(wLC, wRC, fL, fR, P, F);
    } else {
      riemann_tvdmu_hd<T, NDIR>(wLC, wRC, fL, fR, P, F);
    }
  } else if constexpr (SOLVER == SOLVER_TVDLF) {
    st |= cbounds<T, MHD, NDIR, GLM, D, false, BS, FAST>(wLC, wRC, wLp, wRp, P, cmax, cmin);
    riemann_tvdlf<T, NW>(wLC, wRC, fL, fR, cmax, T(P.tvdlfeps), F);
  } else {
    st |= cbounds<T, MHD, NDIR, GLM, D, true, BS, FAST>(wLC, wRC, wLp, wRp, P, cmax, cmin);
    if constexpr (SOLVER == SOLVER_HLL) {
      riemann_hll<T, MHD, NDIR, GLM, NDIM, D, FAST>(wLC, wRC, fL, fR, cmax, cmin, T(P.tvdlfeps), F);
    } else if constexpr (SOLVER == SOLVER_HLLC) {
      if constexpr (MHD) riemann_hllc_mhd<T, NDIR, GLM, NDIM, D, FAST>(wLC, wRC, fL, fR, cmax, cmin, T(P.tvdlfeps), F);
      else riemann_hllc_hd<T, NDIR, D, FAST>(wLC, wRC, fL, fR, cmax, cmin, F);
    } else {
      static_assert(MHD, "HLLD needs MHD");
      riemann_hlld<T, NDIR, GLM, NDIM, D, FAST>(wLC, wRC, wLp, wRp, fL, fR, cmax, cmin, F);
    }
  }
  return st;
}

// MP5 reconstruction (MP5limiter, src/limiter/mod_mp5.t:16-201: Suresh &
// Huynh 1997 in the convention of Mignone et al. 2010), minmod and median as
// mod_mp5.t:404-432.  mp5_side(w(i-2), w(i-1), w(i), w(i+1), w(i+2)) is the
// left state at face i+1/2; the right state is the same formula on the data
// mirrored about the face, mp5_side(w(i+3), w(i+2), w(i+1), w(i), w(i-1)),
// which reproduces the reference's right-side expressions term for term.
__device__ __forceinline__ double mp5_minmod(double a, double b) {
  return (copysign(1.0, a) + copysign(1.0, b)) / 2.0 * fmin(fabs(a), fabs(b));
}
__device__ __forceinline__ double mp5_median(double a, double b, double c) {
  const double t1 = b - a, t2 = c - a;
  return a + (copysign(1.0, t1) + copysign(1.0, t2)) / 2.0 * fmin(fabs(t1), fabs(t2));
}
__device__ __forceinline__ double mp5_side(double wmm, double wm, double w0, double wp, double wpp) {
  const double f = (1.0 / 60.0) * ((((2.0 * wmm - 13.0 * wm) + 47.0 * w0) + 27.0 * wp) - 3.0 * wpp);
  const double b = 4.0 * (w0 - wm);  // alpha = 4
  const double fmp = w0 + mp5_minmod(wp - w0, b);
  const double ful = w0 + b;
  const double dm = (w0 - 2.0 * wm) + wmm;   // d at i-1
  const double d0 = (wp - 2.0 * w0) + wm;    // d at i
  const double dp = (wpp - 2.0 * wp) + w0;   // d at i+1
  const double dm4_0 = mp5_minmod(mp5_minmod(4.0 * d0 - dp, 4.0 * dp - d0), mp5_minmod(d0, dp));
  const double dm4_m = mp5_minmod(mp5_minmod(4.0 * dm - d0, 4.0 * d0 - dm), mp5_minmod(dm, d0));
  const double fmd = (w0 + wp) / 2.0 - dm4_0 / 2.0;
  const double flc = 0.5 * (3.0 * w0 - wm) + (4.0 / 3.0) * dm4_m;
  const double fmin_ = fmax(fmin(fmin(w0, wp), fmd), fmin(fmin(w0, ful), flc));
  const double fmax_ = fmin(fmax(fmax(w0, wp), fmd), fmax(fmax(w0, ful), flc));
  if ((f - w0) * (f - fmp) <= 0.0) return f;
  return mp5_median(fmin_, f, fmax_);
}

// WENO5 family (WENO5limiter, src/limiter/mod_weno.t:254-377; var 1 WENO-JS,
// 2 WENO-Z, 3 WENO-Z+ with lambda = dx^(2/3)): the left state at face i+1/2
// from w(i-2) .. w(i+2); the right state is the same expression on the
// mirrored data, as for MP5.  Constants as the reference writes them.
__device__ __forceinline__ double weno5_side(double wmm, double wm, double w0, double wp, double wpp, int var,
                                             double lambda) {
  constexpr double eps = 1.0e-18;  // weno_eps_machine
  constexpr double b1 = 1.0833333333333333, b2 = 0.25;
  constexpr double d1 = 1.0 / 10.0, d2 = 3.0 / 5.0, d3 = 3.0 / 10.0;
  const double f1 = (1.0 / 3.0) * wmm + (-7.0 / 6.0) * wm + (11.0 / 6.0) * w0;
  const double f2 = (-1.0 / 6.0) * wm + (5.0 / 6.0) * w0 + (1.0 / 3.0) * wp;
  const double f3 = (1.0 / 3.0) * w0 + (5.0 / 6.0) * wp + (-1.0 / 6.0) * wpp;
  const double s1 = wmm + w0 - 2.0 * wm, t1 = wmm - 4.0 * wm + 3.0 * w0;
  const double s2 = wm + wp - 2.0 * w0, t2 = wm - wp;
  const double s3 = w0 + wpp - 2.0 * wp, t3 = 3.0 * w0 - 4.0 * wp + wpp;
  const double be1 = b1 * (s1 * s1) + b2 * (t1 * t1);
  const double be2 = b1 * (s2 * s2) + b2 * (t2 * t2);
  const double be3 = b1 * (s3 * s3) + b2 * (t3 * t3);
  double a1, a2, a3;
  if (var == 1) {
    a1 = d1 / ((be1 + eps) * (be1 + eps));
    a2 = d2 / ((be2 + eps) * (be2 + eps));
    a3 = d3 / ((be3 + eps) * (be3 + eps));
  } else if (var == 2) {
    const double tau = fabs(be1 - be3);
    const double r1 = tau / (be1 + eps), r2 = tau / (be2 + eps), r3 = tau / (be3 + eps);
    a1 = d1 * (1.0 + r1 * r1);
    a2 = d2 * (1.0 + r2 * r2);
    a3 = d3 * (1.0 + r3 * r3);
  } else {
    const double tau = fabs(be1 - be3);
    const double r1 = (tau + eps) / (be1 + eps), r2 = (tau + eps) / (be2 + eps), r3 = (tau + eps) / (be3 + eps);
    a1 = d1 * (1.0 + r1 * r1 + lambda / r1);
    a2 = d2 * (1.0 + r2 * r2 + lambda / r2);
    a3 = d3 * (1.0 + r3 * r3 + lambda / r3);
  }
  const double asum = ((0.0 + a1) + a2) + a3;
  return ((0.0 + f1 * a1 / asum) + f2 * a2 / asum) + f3 * a3 / asum;
}

// WENO3 family (WENO3limiter, src/limiter/mod_weno.t:165-252; var 1 WENO3,
// 2 WENO-YC3 with dx^2 in the weights): the left state at face i+1/2 from
// w(i-1), w(i), w(i+1); the right state on the mirrored data w(i+2), w(i+1),
// w(i) (the smoothness indicators are squares, so the mirror is exact).
__device__ __forceinline__ double weno3_side(double wm, double w0, double wp, int var, double dx2) {
  constexpr double eps = 1.0e-18;  // weno_eps_machine
  const double f1 = (-1.0 / 2.0) * wm + (3.0 / 2.0) * w0;
  const double f2 = (1.0 / 2.0) * w0 + (1.0 / 2.0) * wp;
  const double d1 = w0 - wm, d2 = wp - w0;
  const double be1 = d1 * d1, be2 = d2 * d2;
  double a1, a2;
  if (var == 1) {
    a1 = (1.0 / 3.0) / ((be1 + eps) * (be1 + eps));
    a2 = (2.0 / 3.0) / ((be2 + eps) * (be2 + eps));
  } else {
    const double tau = fabs(be2 - be1);
    a1 = (1.0 / 3.0) * (1.0 + tau / (be1 + dx2));
    a2 = (2.0 / 3.0) * (1.0 + tau / (be2 + dx2));
  }
  const double asum = (0.0 + a1) + a2;
  return (0.0 + f1 * a1 / asum) + f2 * a2 / asum;
}

// Venkatakrishnan's limiter function phi of one cell from w(i-1), w(i),
// w(i+1) (venklimiter, src/limiter/mod_venk.t:6-106; k = 0.3, omega = 1e-12,
// eps2 = (k dx)^3).
__device__ __forceinline__ double venk_phi(double wm, double w0, double wp, double eps2) {
  constexpr double omega = 1.0e-12;
  const double wmax = fmax(fmax(wm, w0), wp), wmin = fmin(fmin(wm, w0), wp);
  const double westp = w0 + (wp - wm) * 0.25, westm = w0 - (wp - wm) * 0.25;
  auto ratio = [&](double dp, double dmr) {
    const double dm = copysign(fabs(dmr) + omega, dmr);
    const double p1 = (dp * dp + eps2) + 2.0 * dp * dm;
    const double p2 = ((dp * dp + 2.0 * (dm * dm)) + dp * dm) + eps2;
    return p1 / p2;
  };
  double phip = 1.0, phim = 1.0;
  if (westp > w0) phip = ratio(wmax - w0, westp - w0);
  else if (westp < w0) phip = ratio(wmin - w0, westp - w0);
  if (westm < w0) phim = ratio(-(wmax - w0), westm - w0);
  else if (westm > w0) phim = ratio(-(wmin - w0), westm - w0);
  return fmin(phim, phip);
}

// Halo width of the staged tile: two cells for the slope limiters, three for
// the fifth-order reconstructions (face stencil i-2 .. i+3).  LIM_WENO5 as a
// template argument stands for the whole WENO5 family (variant at run time).
template <int LIM>
struct HaloW {
  static constexpr int value = (LIM == LIM_MP5 || LIM == LIM_WENO5) ? 3 : 2;
};

// Shared-memory tile of BN x BN cells (sizes in doubles), halo width HW.
template <class TF, int NW, int NDIM, int HW = 2, int BN = BN16>
struct Tile {
  static constexpr int H2 = 2 * HW;
  static constexpr int NSLOT = NDIM == 3 ? H2 : 1;      // z ring: planes k-HW+1 .. k+HW
  static constexpr int PLANE = BN * BN;
  static constexpr int RING = NSLOT * NW * PLANE;        // [slot][v][j][i]
  static constexpr int HX = NW * BN * H2;                // [v][j][c] c: i=-HW..-1, BN..BN+HW-1
  static constexpr int HY = NW * H2 * BN;                // [v][r][i] r: j likewise
  static constexpr int HC = NW * H2 * H2;                // [v][r][c] corners
  static constexpr int FB = NW * (BN + 1) * BN;          // [v][face]
  static constexpr int YX = NW * BN;                     // [v][i] y-faces of the top row (j = BN)
  static constexpr int TOTAL = RING + HX + HY + HC + FB + YX;
  static constexpr size_t BYTES = sizeof(TF) * TOTAL;
};

template <int HW, int BN = BN16>
__device__ __forceinline__ int halo_slot_w(int c) { return c < 0 ? c + HW : c - (BN - HW); }

// Ring slot of z-plane k (k >= -2 HW).
template <int HW>
__device__ __forceinline__ int ring_slot(int k) {
  if constexpr (HW == 2) return k & 3;
  else return (k + 4 * HW) % (2 * HW);
}

template <class TF, int NW, int NDIM, int HW = 2, int BN = BN16>
struct TileView {
  static constexpr int H2 = 2 * HW;
  TF *ring, *hx, *hy, *hc, *fb, *yx;
  __device__ TileView(TF *s) {
    using T = Tile<TF, NW, NDIM, HW, BN>;
    ring = s;
    hx = ring + T::RING;
    hy = hx + T::HX;
    hc = hy + T::HY;
    fb = hc + T::HC;
    yx = fb + T::FB;
  }
  // primitive v at in-plane (i, j) in [-HW, BN+HW-1]^2 of the plane held in `slot`
  __device__ __forceinline__ TF at(int slot, int v, int i, int j) const {
    const bool ii = (unsigned)i < (unsigned)BN, jj = (unsigned)j < (unsigned)BN;
    if (ii && jj) return ring[(slot * NW + v) * (BN * BN) + j * BN + i];
    if (jj) return hx[(v * BN + j) * H2 + halo_slot_w<HW, BN>(i)];
    if (ii) return hy[(v * H2 + halo_slot_w<HW, BN>(j)) * BN + i];
    return hc[(v * H2 + halo_slot_w<HW, BN>(j)) * H2 + halo_slot_w<HW, BN>(i)];
  }
  // Offset (in doubles from the tile start) of variable 0 at in-plane (i, j)
  // of the plane in `slot`, and the stride between variables there; branch-free.
  __device__ __forceinline__ void addr(int slot, int i, int j, int &base, int &stride) const {
    using T = Tile<TF, NW, NDIM, HW, BN>;
    const bool ii = (unsigned)i < (unsigned)BN, jj = (unsigned)j < (unsigned)BN;
    const int hi = halo_slot_w<HW, BN>(i), hj = halo_slot_w<HW, BN>(j);
    const int oc = slot * NW * (BN * BN) + j * BN + i;
    const int ox = T::RING + j * H2 + hi;
    const int oy = T::RING + T::HX + hj * BN + i;
    const int oz = T::RING + T::HX + T::HY + hj * H2 + hi;
    base = ii ? (jj ? oc : oy) : (jj ? ox : oz);
    stride = ii ? (jj ? BN * BN : H2 * BN) : (jj ? H2 * BN : H2 * H2);
  }
  __device__ __forceinline__ TF &center(int slot, int v, int i, int j) {
    return ring[(slot * NW + v) * (BN * BN) + j * BN + i];
  }
};

// Runtime form of orig_index for a face phase D (the v loop is unrolled, so
// only D is a run-time value: a few integer operations per variable).
template <bool MHD, int NDIR>
__device__ __forceinline__ int orig_index_rt(int v, int D) {
  if (v >= 1 && v <= NDIR) return 1 + (v - 1 + D) % NDIR;
  if (MHD && v >= NDIR + 2 && v <= 2 * NDIR + 1) return NDIR + 2 + (v - NDIR - 2 + D) % NDIR;
  return v;
}

// TF: arithmetic type of the face computation — double (plain FP64 path) or
// float (mixed form: reconstruction, wave speeds, fluxes and Riemann solver in
// FP32; conserved state, pressure recovery, RK algebra, flux-divergence
// accumulation, sources and the small-value fix of wnew in FP64).
// Mixed form, cold path: a face whose FP32 flux came out non-finite (FP32
// round-off in a near-degenerate star state of a strong jump, e.g. the HLLD
// denominator rho (S - u)(S - S_M) - Bn^2) is recomputed in FP64 from the
// same staged primitives: reconstruction and Riemann flux as the FP64 kernel
// does them.  It runs in a fix-up pass after the face phase, only when some
// face of the phase failed, and out of line, so the hot face loop keeps its
// registers; the flux comes back by value (rotated order, like the FP32 one).
template <int NW>
struct FaceFlux64 {
  double F[NW];
  uint32_t st;
};

template <class TF, bool MHD, int NDIR, bool GLM, int NDIM, int SOLVER, int LIM, int BS>
__device__ __noinline__ FaceFlux64<Vars<MHD, NDIR, GLM>::NW> face_retry_fp64(
    const TF *smem, int D, int b0, int b1, int b2, int b3, int s0, int s1, int s2, int s3, double rd, double cg,
    const PhysParams P) {
  using V = Vars<MHD, NDIR, GLM>;
  constexpr int NW = V::NW;
  const int base[4] = {b0, b1, b2, b3}, strd[4] = {s0, s1, s2, s3};
  double wLp[NW], wRp[NW];
#pragma unroll
  for (int v = 0; v < NW; ++v) {
    const int ov = orig_index_rt<MHD, NDIR>(v, D);
    double q[4];
#pragma unroll
    for (int o = 0; o < 4; ++o) q[o] = double(smem[base[o] + ov * strd[o]]);
    const double d0 = q[1] - q[0], d1 = q[2] - q[1], d2 = q[3] - q[2];
    double ldw, rdw;
    face_slopes<double, LIM>(P.limiter, d0, d1, d2, rd, ldw, rdw);
    wLp[v] = q[1] + 0.5 * ldw;
    wRp[v] = q[2] - 0.5 * rdw;
  }
  FaceFlux64<NW> r;
  r.st = face_from_states<double, MHD, NDIR, GLM, NDIM, SOLVER, BS>(wLp, wRp, P, cg, r.F);
  return r;
}

// Mixed form's recomputation: the face's four stencil cells (R cell at
// block-local (i, j, k), the others 2 and 1 below it and 1 above along D)
// gathered from the FP64 state and converted exactly as the FP64 kernel
// stages them (load_prim), then the guarded FP64 reconstruction, small-value
// check and Riemann flux: a recomputed face carries the FP64 kernel's flux
// and its FP64 small-value decisions.  The staged cells' own status bits
// were raised when they were staged.
template <bool MHD, int NDIR, bool GLM, int NDIM, int SOLVER, int LIM, int BS, int BN>
__device__ __noinline__ FaceFlux64<Vars<MHD, NDIR, GLM>::NW> face_retry_state(const StageArgs *A, int b, int D, int i,
                                                                             int j, int k, double rd, double cg) {
  using V = Vars<MHD, NDIR, GLM>;
  constexpr int NW = V::NW;
  double q[4][NW];
#pragma unroll
  for (int o = 0; o < 4; ++o)
    load_prim<MHD, NDIR, GLM, NDIM, BN>(*A, b, i + (D == 0 ? o - 2 : 0), j + (D == 1 ? o - 2 : 0),
                                        k + (D == 2 ? o - 2 : 0), q[o]);
  double wLp[NW], wRp[NW];
#pragma unroll
  for (int v = 0; v < NW; ++v) {
    const int ov = orig_index_rt<MHD, NDIR>(v, D);
    const double d0 = q[1][ov] - q[0][ov], d1 = q[2][ov] - q[1][ov], d2 = q[3][ov] - q[2][ov];
    double ldw, rdw;
    face_slopes<double, LIM>(A->P.limiter, d0, d1, d2, rd, ldw, rdw);
    wLp[v] = q[1][ov] + 0.5 * ldw;
    wRp[v] = q[2][ov] - 0.5 * rdw;
  }
  FaceFlux64<NW> r;
  r.st = face_from_states<double, MHD, NDIR, GLM, NDIM, SOLVER, BS>(wLp, wRp, A->P, cg, r.F);
  return r;
}

// The mixed form's small-value decisions are made in FP64: with
// fix_small_values set, a face whose FP32 left or right state has a density
// or pressure within 2^-14 of its stencil's largest magnitude of the floor
// (or below it) is recomputed by face_retry_state.  The FP32 state differs
// from the FP64 one by a few FP32 roundings of that magnitude (2^-21 at
// most), so every face the FP64 check would flag is recomputed.
template <bool MHD, int NDIR, bool GLM>
__device__ __forceinline__ bool sv_near_floor(const float *wLp, const float *wRp, float srho, float sp,
                                              const PhysParams &P) {
  using V = Vars<MHD, NDIR, GLM>;
  const float m = 0x1p-14f;
  return wLp[V::RHO] < float(P.small_density) + m * srho || wRp[V::RHO] < float(P.small_density) + m * srho ||
         wLp[V::E] < float(P.small_pressure) + m * sp || wRp[V::E] < float(P.small_pressure) + m * sp;
}

// MUSCL-Hancock predictor, one direction D (hancock, src/mod_finite_volume.t:
// 56-101; reconstruct_LR default branch 1171-1222): from the primitives of
// cells c-1, c, c+1 along D (shared-memory offsets base[o], strides strd[o]),
// the cell's limited edge states — right edge wprim + ldw/2 (the left state of
// the face above), left edge wprim - rdw/2 (the right state of the face
// below) — the primitive small-value check on both, their conserved forms and
// physical fluxes, and wnew += -qdt/dx (f(right edge) - f(left edge)).  No
// Riemann solver and no GLM state modification.  D is a template parameter
// so the accumulator index stays compile-time (registers, no local memory).
template <bool MHD, int NDIR, bool GLM, int LIM, int D>
__device__ __forceinline__ uint32_t hancock_dir(const double *smem, const int *base, const int *strd, double rd,
                                                double sc, double cg, const PhysParams &P, double *acc) {
  using V = Vars<MHD, NDIR, GLM>;
  constexpr int NW = V::NW;
  double wl[NW], wr[NW];
#pragma unroll
  for (int v = 0; v < NW; ++v) {
    const int ov = orig_index<MHD, NDIR, D>(v);
    const double q0 = smem[base[0] + ov * strd[0]], q1 = smem[base[1] + ov * strd[1]],
                 q2 = smem[base[2] + ov * strd[2]];
    const double dm = q1 - q0, dp = q2 - q1;
    wr[v] = q1 + 0.5 * limited_slope<double, true, LIM>(P.limiter, dp, dm, rd);
    wl[v] = q1 - 0.5 * limited_slope<double, false, LIM>(P.limiter, dp, dm, rd);
  }
  uint32_t st = 0;
  if (P.fix_small_values) {
    const bool fr = small_values<double, MHD, NDIR, GLM>(wr, true, P);
    const bool fl = small_values<double, MHD, NDIR, GLM>(wl, true, P);
    if ((fr || fl) && P.small_values_method != 1) st |= ST_SMALL_VALUE;
  }
  double cl[NW], cr[NW];
#pragma unroll
  for (int v = 0; v < NW; ++v) { cl[v] = wl[v]; cr[v] = wr[v]; }
  to_conserved<double, MHD, NDIR, GLM>(cl, P);
  to_conserved<double, MHD, NDIR, GLM>(cr, P);
  double fl[NW], fr[NW];
  phys_flux<double, MHD, NDIR, GLM, 0>(cl, wl, cg, fl);
  phys_flux<double, MHD, NDIR, GLM, 0>(cr, wr, cg, fr);
#pragma unroll
  for (int v = 0; v < NW; ++v) {
    const int ov = orig_index<MHD, NDIR, D>(v);
    acc[ov] = acc[ov] + sc * (fr[v] - fl[v]);
  }
  return st;
}

// MP5 (three-cell halo) takes one CTA per SM: its 6-plane ring fills most of
// the shared memory of the 3-D MHD tile, and the registers it frees avoid
// spills in the 6-cell face stencil.
// CTAs per SM the stage kernel is built for: two of 256 threads (FP64; one
// with the fifth-order halo), three in the mixed form; smaller tiles keep the
// same threads per SM.
//
// Variants (VAR > 0) are the alternatives the autotuner times for the
// benchmark schemes: threads per CTA, the CTAs per SM the registers are
// capped for, and the staging mode (asynchronous bulk copies of the next
// conserved plane, FP64 only).  stage_variant(VAR, fp64) gives them.
struct StageVariant {
  int threads, minb;
  bool async;
};
__host__ __device__ constexpr StageVariant stage_variant(int var, bool fp64) {
  if (fp64) {
    return var == 1 ? StageVariant{256, 2, true}
                    : var == 2 ? StageVariant{288, 2, false} : StageVariant{256, 1, false};
  }
  return var == 1 ? StageVariant{256, 2, false} : var == 2 ? StageVariant{256, 4, false} : StageVariant{288, 3, false};
}
template <class TF, int LIM, int BN, int VAR = 0>
struct StageOcc {
  static constexpr bool FP64 = sizeof(TF) == 8;
  static constexpr int THREADS =
      VAR > 0 ? stage_variant(VAR, FP64).threads : (BN == BN16 ? STAGE_THREADS : stage_threads(BN));
  static constexpr int BASE = FP64 ? (HaloW<LIM>::value == 3 ? 1 : AMRVAC_STAGE_MINB) : AMRVAC_STAGE_MINB_MIXED;
  static constexpr int MINB0 = BASE * 256 / THREADS < 1 ? 1 : (BASE * 256 / THREADS > 16 ? 16 : BASE * 256 / THREADS);
  static constexpr int MINB = VAR > 0 ? stage_variant(VAR, FP64).minb : MINB0;
  static constexpr bool ASYNC = VAR > 0 && stage_variant(VAR, FP64).async;
};

// Asynchronous plane staging: one thread copies a block's conserved plane
// (TB x TB doubles per variable, contiguous in HBM) into a ring slot with
// bulk copies (cp.async.bulk, this GPU's own memory, no multicast) that
// complete on an mbarrier; the waits are bounded (AMRVAC_ASYNC_SPINS polls)
// and a wait that runs out raises ST_TIMEOUT.
#ifndef AMRVAC_ASYNC_SPINS
#define AMRVAC_ASYNC_SPINS (1 << 22)
#endif
__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint32_t mbar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar) : "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
// n copies of `bytes` each, source stride sstride doubles, destination
// stride dstride bytes; the arrival carries the expected byte count.
__device__ __forceinline__ void plane_copy_async(uint32_t mbar, uint32_t dst, uint32_t dstride, const double *src,
                                                 size_t sstride, int n, uint32_t bytes) {
  // earlier generic-proxy reads of the slot before the asynchronous writes
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(bytes * (uint32_t)n)
               : "memory");
  for (int v = 0; v < n; ++v)
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     dst + (uint32_t)v * dstride),
                 "l"(src + (size_t)v * sstride), "r"(bytes), "r"(mbar)
                 : "memory");
}
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity, int spins = AMRVAC_ASYNC_SPINS) {
  for (int i = 0; i < spins; ++i) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(done)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

template <class TF, bool MHD, int NDIR, bool GLM, int NDIM, int SOLVER, int LIM, int BS, int BN = BN16, int VAR = 0>
__global__ void __launch_bounds__(StageOcc<TF, LIM, BN, VAR>::THREADS, StageOcc<TF, LIM, BN, VAR>::MINB)
    fv_stage_kernel(const __grid_constant__ StageArgs A) {
  using V = Vars<MHD, NDIR, GLM>;
  constexpr int NW = V::NW;
  // block edge BN; this CTA's tile is TB x TB cells of a z-plane (x/y), at
  // (ti0, tj0) in the block; TBY = TB in 2-D and 3-D
  constexpr int TB = tile_edge(BN);
  constexpr int NTX = BN / TB;                       // tiles per plane row
  constexpr int NT = NDIM >= 2 ? NTX * NTX : NTX;    // tiles per plane
  constexpr int THREADS = StageOcc<TF, LIM, BN, VAR>::THREADS;
  constexpr int FB = (TB + 1) * TB;  // face-buffer stride per variable
  constexpr bool FP64 = sizeof(TF) == 8;
  constexpr int HW = HaloW<LIM>::value;  // halo width: 2, or 3 for MP5
  constexpr int H2 = 2 * HW;
  // Faces of the slope limiters use the fast division, reciprocal and square
  // root (physics.cuh: unguarded Newton in FP64, the hardware approximations
  // in the mixed form's FP32); a face whose flux is not finite is recomputed
  // in FP64 with the guarded forms in the fix-up pass after its phase.
  constexpr bool FASTF = !(LIM == LIM_MP5 || LIM == LIM_WENO5 || LIM == LIM_WENO3 || LIM == LIM_VENK);
  constexpr bool RETRY = !FP64 || FASTF;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  TF *smem = reinterpret_cast<TF *>(smem_raw);
  TileView<TF, NW, NDIM, HW, TB> tv(smem);
  const int t = threadIdx.x;
  // Work: global tile-planes g = (block*NT + tile)*PL + k (PL = BN in 3-D,
  // 1 in 2-D).  zchunk > 0: one z-chunk of one tile column per CTA.
  // zchunk == 0: persistent plane ranges — the grid is one wave of CTAs,
  // each marching a contiguous range of tile-planes across block boundaries
  // and re-staging halo planes only where a new tile column starts.
  constexpr int PL = NDIM == 3 ? BN : 1;
  long g, gend;
  if (A.zchunk > 0) {
    const int nchunk = NDIM == 3 ? BN / A.zchunk : 1;
    const int c0 = blockIdx.x / nchunk;  // tile column: block*NT + tile
    if (c0 >= A.nblocks * NT) return;
    g = (long)c0 * PL + (NDIM == 3 ? (blockIdx.x - c0 * nchunk) * A.zchunk : 0);
    gend = g + (NDIM == 3 ? A.zchunk : 1);
  } else {
    const long total = (long)A.nblocks * NT * PL;
    g = (long)blockIdx.x * total / gridDim.x;
    gend = (long)(blockIdx.x + 1) * total / gridDim.x;
  }

  const PhysParams &P = A.P;
  const double dt = *A.dt_dev;
  const double qdt = A.dtfactor * dt;
  const int dsel = sweep_dir(A.sweep, A.split_xy, A.dt_dev, NDIM);  // -1: all directions
  const double cg = GLM ? *A.cmax_dev : 0.0;
  uint32_t st = 0;
  const int ci = t % TB, cj = t / TB;  // cell role (tile-relative) for t < TB*TB
  const bool cell_thread = t < TB * TB;
  const bool need_corners = MHD && !GLM && P.divb == DIVB_LINDE;
  __shared__ int s_retry;  // some face of this phase needs the guarded FP64 recomputation
  if (t == 0) s_retry = 0;
  // Asynchronous staging (variant; 3-D FP64, whole-plane tiles, slope
  // limiters): the conserved plane k+2 that iteration k stages is a
  // contiguous row of TB*TB doubles per variable, in this block or its
  // same-level z neighbour.  One thread copies it into its ring slot at the
  // start of the iteration; the cells convert it to primitives in place
  // just before the z phase, the first phase that reads it, so the copy runs
  // behind the x and y phases.  Planes behind a physical boundary or a level
  // jump take the gather (load_prim).
  constexpr bool ASYNC = StageOcc<TF, LIM, BN, VAR>::ASYNC && FP64 && NDIM == 3 && NT == 1 && HW == 2 &&
                         SOLVER != SOLVER_HANCOCK;
  __shared__ __align__(8) unsigned long long s_mbar;
  uint32_t mphase = 0;
  if constexpr (ASYNC) {
    if (t == 0) mbar_init(smem_addr(&s_mbar));
  }
#pragma unroll 1
  while (g < gend) {
  const int col = (int)(g / PL);  // tile column: block*NT + tile
  const int b = col / NT;
  const int ti0 = NT == 1 ? 0 : ((col - b * NT) % NTX) * TB;   // tile origin in the block
  const int tj0 = NT == 1 ? 0 : ((col - b * NT) / NTX) * TB;
  const int bi = ti0 + ci, bj = NDIM >= 2 ? tj0 + cj : 0;      // the cell role's cell in the block
  const int k0 = (int)(g - (long)col * PL);
  const int k1 = (int)(k0 + ((gend - g) < (PL - k0) ? (gend - g) : (PL - k0)));
  g += k1 - k0;
  uint32_t stb = 0;  // status of this block's update
  const int amr_mask = A.amr_face ? A.amr_face[b] : 0;
  double dx[3], dxinv[3], rdel[3];
  [[maybe_unused]] double wlam[3];  // WENO-Z+: dx^(2/3) per direction
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    dx[d] = d < NDIM ? A.dxb[b * 3 + d] : 1.0;
    dxinv[d] = -qdt / dx[d];
    const double r = P.cada3_radius * dx[d];
    // cada3: 1 / (cada3_radius dx)^2; schmid: (a2max + cadepsilon) dx^2 with
    // a2max = schmid_rad (schmid2) or a2max_global of this step (schmid1)
    const double a2m = P.schmid_global ? A.dt_dev[10 + d] : P.schmid_rad[d];
    rdel[d] = (LIM == LIM_SCHMID || (LIM == 0 && P.limiter == LIM_SCHMID))
                  ? (a2m + 1.0e-14) * (dx[d] * dx[d]) : 1.0 / (r * r);
    if constexpr (LIM == LIM_WENO5) wlam[d] = pow(dx[d], 2.0 / 3.0);
  }
  double fz_prev[NDIM == 3 ? NW : 1];
#pragma unroll
  for (int v = 0; v < (NDIM == 3 ? NW : 1); ++v) fz_prev[v] = 0.0;

  // 3-D: iteration k stages plane k+HW; iterations k0-2HW .. k0-1 only stage
  // the planes k0-HW .. k0+HW-1 (and, at k0-1, compute the z-face k0-1/2);
  // iterations k0 .. k1-1 update plane k.
  const int kstart = NDIM == 3 ? k0 - 2 * HW : 0;
#pragma unroll 1
  for (int k = kstart; k < k1; ++k) {
    const bool update = k >= k0;
    const int slot = NDIM == 3 ? ring_slot<HW>(k) : 0;
    // ---- stage plane k+HW (3-D) / the block (2-D) as primitives
    bool pend = false;  // an asynchronous copy of plane k+HW is in flight (uniform)
    if constexpr (ASYNC) {
      const int kk = k + HW;
      int src = b, sk = kk;
      if (kk >= BN || kk < 0) {  // the z neighbour's plane, if it is a same-level block
        src = A.nbr[b * 27 + dir_index(0, 0, kk >= BN ? 1 : -1)];
        sk = kk >= BN ? kk - BN : kk + BN;
      }
      if (src >= 0 && src < A.nblocks) {
        pend = true;
        if (t == 0)
          plane_copy_async(smem_addr(&s_mbar), smem_addr(&tv.center(ring_slot<HW>(kk), 0, 0, 0)),
                           (uint32_t)(sizeof(double) * TB * TB), A.uin + cell_offset<3>(src, NW, 0, 0, 0, sk, BN),
                           (size_t)BN * BN * BN, NW, (uint32_t)(sizeof(double) * TB * TB));
      }
    }
    if (cell_thread && !pend) {
      double w[NW];
      const int kk = NDIM == 3 ? k + HW : 0;
      stb |= load_prim<MHD, NDIR, GLM, NDIM, BN>(A, b, bi, bj, kk, w);
      const int s2 = NDIM == 3 ? ring_slot<HW>(kk) : 0;
#pragma unroll
      for (int v = 0; v < NW; ++v) tv.center(s2, v, ci, cj) = TF(w[v]);
    }
    // the asynchronous plane: wait for the copy (bounded) and convert each
    // cell to primitives in place, with load_prim's small-value check
    auto finish_async = [&]() {
      if constexpr (ASYNC) {
        if (!mbar_wait(smem_addr(&s_mbar), mphase)) {
          stb |= ST_TIMEOUT;
          mbar_wait(smem_addr(&s_mbar), mphase);  // a second bounded wait for the copy in flight
        }
        mphase ^= 1u;
        if (cell_thread) {
          const int s2 = ring_slot<HW>(k + HW);
          double w[NW];
#pragma unroll
          for (int v = 0; v < NW; ++v) w[v] = double(tv.center(s2, v, ci, cj));
          if (P.fix_small_values) {
            if (small_values<double, MHD, NDIR, GLM>(w, false, P) && P.small_values_method != 1) stb |= ST_SMALL_VALUE;
          }
          to_primitive<MHD, NDIR, GLM>(w, P);
#pragma unroll
          for (int v = 0; v < NW; ++v) tv.center(s2, v, ci, cj) = TF(w[v]);
        }
      }
      pend = false;
    };
    // ---- x/y halo strips (and corners for Linde) of plane k
    constexpr int NHX = TB * H2, NHY = H2 * TB, NHC = H2 * H2;
    const int nhalo = update ? (need_corners ? NHX + NHY + NHC : NHX + NHY) : 0;
    // (small tiles have fewer threads than halo cells: a thread may take two)
#pragma unroll 1
    for (int h = t; h < nhalo; h += THREADS) {
      int i, j, stride;
      TF *dst;
      if (h < NHX) {
        j = h / H2;
        const int c = h - j * H2;
        i = c < HW ? c - HW : c + TB - HW;
        dst = tv.hx + j * H2 + c;
        stride = TB * H2;
      } else if (h < NHX + NHY) {
        const int r = (h - NHX) / TB;
        i = (h - NHX) - r * TB;
        j = r < HW ? r - HW : r + TB - HW;
        dst = tv.hy + r * TB + i;
        stride = H2 * TB;
      } else {
        const int r = (h - NHX - NHY) / H2, c = (h - NHX - NHY) - r * H2;
        i = c < HW ? c - HW : c + TB - HW;
        j = r < HW ? r - HW : r + TB - HW;
        dst = tv.hc + r * H2 + c;
        stride = H2 * H2;
      }
      double w[NW];
      stb |= load_prim<MHD, NDIR, GLM, NDIM, BN>(A, b, i + ti0, j + tj0, k, w);
#pragma unroll
      for (int v = 0; v < NW; ++v) dst[v * stride] = TF(w[v]);
    }
    // ---- RK combination wnew0 = a*base + b*in (src/mod_advance.t:254-266)
    double acc[NW];
    if (update && cell_thread) {
#pragma unroll
      for (int v = 0; v < NW; ++v) {
        const size_t o = cell_offset<NDIM>(b, NW, v, bi, bj, k, BN);
        const double win = A.uin[o];
        acc[v] = (A.a_base == 0.0) ? win : A.a_base * A.ubase[o] + A.b_in * win;
      }
    }
    __syncthreads();
    if constexpr (SOLVER == SOLVER_HANCOCK) {
      // ---- Hancock predictor: each cell thread, all directions, from the
      // staged primitives (cells c-1, c, c+1; z from ring slots k-1..k+1)
      static_assert(sizeof(TF) == 8, "the Hancock predictor is FP64 only");
      if (update && cell_thread) {
        int base[3], strd[3];
        if (dsel < 0 || dsel == 0) {
#pragma unroll
          for (int o = 0; o < 3; ++o) tv.addr(slot, ci + o - 1, cj, base[o], strd[o]);
          stb |= hancock_dir<MHD, NDIR, GLM, LIM, 0>(smem, base, strd, rdel[0], dxinv[0], cg, P, acc);
        }
        if (dsel < 0 || dsel == 1) {
#pragma unroll
          for (int o = 0; o < 3; ++o) tv.addr(slot, ci, cj + o - 1, base[o], strd[o]);
          stb |= hancock_dir<MHD, NDIR, GLM, LIM, 1>(smem, base, strd, rdel[1], dxinv[1], cg, P, acc);
        }
        if (NDIM == 3 && (dsel < 0 || dsel == 2)) {
#pragma unroll
          for (int o = 0; o < 3; ++o) {
            base[o] = ring_slot<HW>(k + o - 1) * NW * (TB * TB) + cj * TB + ci;
            strd[o] = TB * TB;
          }
          stb |= hancock_dir<MHD, NDIR, GLM, LIM, 2>(smem, base, strd, rdel[2], dxinv[2], cg, P, acc);
        }
      }
    } else {
    // ---- face phases x, y (plane k) and z (face k+1/2 of every column); one
    // copy of the face code serves all three through the state rotation.
    // The x phase also computes the 16 y-faces of the top row (j = BN) into
    // tv.yx: 272 x-faces + 16 = 288 faces make its second round one full warp,
    // and the y phase one round of 256 (instead of two rounds of 256 + 16).
    // (With 272 or more threads a phase of 272 faces is one round already;
    // a split sweep has one phase only.)
    const bool merge_yx = THREADS < FB && dsel < 0;
    const int dlo = update ? 0 : (NDIM == 3 && k == k0 - 1 ? 2 : NDIM);
#pragma unroll 1
    for (int D = dlo; D < NDIM; ++D) {
      if (pend && D == 2) {  // the z phase reads plane k+2 (k+HW)
        finish_async();
        __syncthreads();
      }
      if (dsel >= 0 && D != dsel) continue;  // not this sweep's direction (uniform)
      const int nface = D == 0 ? (merge_yx ? FB + TB : FB) : (D == 1 && !merge_yx ? FB : TB * TB);
      // direction FD and index fl (in that direction's face layout) of face f
      // of this phase
      auto face_dir = [&](int f, int &FD, int &fl) {
        if (merge_yx && D == 0 && f >= FB) { FD = 1; fl = TB * TB + (f - FB); }
        else { FD = D; fl = f; }
      };
      // where the flux of variable ov of face f lives
      auto flux_ref = [&](int f, int FD, int fl, int ov) -> TF & {
        return FD == D ? tv.fb[ov * FB + f] : tv.yx[ov * TB + (fl - TB * TB)];
      };
      // face coordinates and the shared-memory offsets of the 2 HW stencil
      // cells (variable 0) with the per-variable strides
      auto face_at = [&](int FD, int fl, int &fi, int &fj, int *base, int *strd) {
        if (FD == 0) { fj = fl / (TB + 1); fi = fl - fj * (TB + 1); }
        else { fj = fl / TB; fi = fl - fj * TB; }
#pragma unroll
        for (int o = 0; o < H2; ++o) {
          if (FD == 2) {
            base[o] = ring_slot<HW>(k + o - HW + 1) * NW * (TB * TB) + fl;
            strd[o] = TB * TB;
          } else {
            tv.addr(slot, FD == 0 ? fi + o - HW : fi, FD == 0 ? fj : fj + o - HW, base[o], strd[o]);
          }
        }
      };
      // level jump across this block face: keep the boundary face flux
      // (store_flux, src/mod_fix_conserve.t:597-648) for the flux fix
      auto capture = [&](int FD, int fi, int fj, const TF *Fr, double sc) {
        const int pos = FD == 0 ? fi + ti0 : (FD == 1 ? fj + tj0 : k + 1);  // face position in the block
        const int side = pos == 0 ? 0 : (pos == BN ? 1 : -1);
        if (side >= 0 && ((amr_mask >> (2 * FD + side)) & 1)) {
          const int ta = FD == 0 ? fj + tj0 : fi + ti0, tb = FD == 2 ? fj + tj0 : k;
          double *pf = A.pflux + ((size_t)A.gslot[b] * (2 * NDIM) + 2 * FD + side) * NW * (BN * BN);
#pragma unroll
          for (int v = 0; v < NW; ++v)
            pf[orig_index_rt<MHD, NDIR>(v, FD) * (BN * BN) + ta + BN * (NDIM == 3 ? tb : 0)] = sc * double(Fr[v]);
        }
      };
#pragma unroll 1
      for (int f = t; f < nface; f += THREADS) {
        int fi, fj, FD, fl;
        face_dir(f, FD, fl);
        const TF rd = TF(FD == 0 ? rdel[0] : (FD == 1 ? rdel[1] : rdel[2]));
        TF wLp[NW], wRp[NW];
        int base[H2], strd[H2];
        face_at(FD, fl, fi, fj, base, strd);
        if constexpr (LIM == LIM_MP5) {
          static_assert(FP64, "MP5 is FP64 only");
          // MP5limiter, then fix_limiter1 (src/limiter/mod_weno.t:135-163):
          // a variable keeps the flat states w(i), w(i+1) where phys_check_w
          // flags it (rho < small_density, p < small_pressure) in either
          // reconstructed state
#pragma unroll
          for (int v = 0; v < NW; ++v) {
            const int ov = orig_index_rt<MHD, NDIR>(v, FD);
            double q[6];
#pragma unroll
            for (int o = 0; o < 6; ++o) q[o] = smem[base[o] + ov * strd[o]];
            wLp[v] = mp5_side(q[0], q[1], q[2], q[3], q[4]);
            wRp[v] = mp5_side(q[5], q[4], q[3], q[2], q[1]);
          }
          // density and energy are not rotated: variable index = tile index
          if (wLp[V::RHO] < P.small_density || wRp[V::RHO] < P.small_density) {
            wLp[V::RHO] = smem[base[2] + V::RHO * strd[2]];
            wRp[V::RHO] = smem[base[3] + V::RHO * strd[3]];
          }
          if (wLp[V::E] < P.small_pressure || wRp[V::E] < P.small_pressure) {
            wLp[V::E] = smem[base[2] + V::E * strd[2]];
            wRp[V::E] = smem[base[3] + V::E * strd[3]];
          }
        } else if constexpr (LIM == LIM_WENO5) {
          static_assert(FP64, "WENO5 is FP64 only");
          // WENO5limiter, then fix_limiter (src/limiter/mod_weno.t:100-133): a
          // flagged density or pressure in either state makes every variable
          // of the face take the flat states w(i), w(i+1)
          const int var = P.limiter == LIM_WENO5 ? 1 : (P.limiter == LIM_WENOZ5 ? 2 : 3);
          const double lam = FD == 0 ? wlam[0] : (FD == 1 ? wlam[1] : wlam[2]);
#pragma unroll
          for (int v = 0; v < NW; ++v) {
            const int ov = orig_index_rt<MHD, NDIR>(v, FD);
            double q[6];
#pragma unroll
            for (int o = 0; o < 6; ++o) q[o] = smem[base[o] + ov * strd[o]];
            wLp[v] = weno5_side(q[0], q[1], q[2], q[3], q[4], var, lam);
            wRp[v] = weno5_side(q[5], q[4], q[3], q[2], q[1], var, lam);
          }
          if (wLp[V::RHO] < P.small_density || wRp[V::RHO] < P.small_density || wLp[V::E] < P.small_pressure ||
              wRp[V::E] < P.small_pressure) {
#pragma unroll
            for (int v = 0; v < NW; ++v) {
              const int ov = orig_index_rt<MHD, NDIR>(v, FD);
              wLp[v] = smem[base[2] + ov * strd[2]];
              wRp[v] = smem[base[3] + ov * strd[3]];
            }
          }
        } else if constexpr (LIM == LIM_WENO3) {
          static_assert(FP64, "WENO3 is FP64 only");
          // WENO3limiter then fix_limiter (all variables flat where density or
          // pressure is flagged in either state)
          const int var = P.limiter == LIM_WENO3 ? 1 : 2;
          const double dxd = FD == 0 ? dx[0] : (FD == 1 ? dx[1] : dx[2]);
          const double dx2 = dxd * dxd;
#pragma unroll
          for (int v = 0; v < NW; ++v) {
            const int ov = orig_index_rt<MHD, NDIR>(v, FD);
            double q[4];
#pragma unroll
            for (int o = 0; o < 4; ++o) q[o] = smem[base[o] + ov * strd[o]];
            wLp[v] = weno3_side(q[0], q[1], q[2], var, dx2);
            wRp[v] = weno3_side(q[3], q[2], q[1], var, dx2);
          }
          if (wLp[V::RHO] < P.small_density || wRp[V::RHO] < P.small_density || wLp[V::E] < P.small_pressure ||
              wRp[V::E] < P.small_pressure) {
#pragma unroll
            for (int v = 0; v < NW; ++v) {
              const int ov = orig_index_rt<MHD, NDIR>(v, FD);
              wLp[v] = smem[base[1] + ov * strd[1]];
              wRp[v] = smem[base[2] + ov * strd[2]];
            }
          }
        } else if constexpr (LIM == LIM_VENK) {
          static_assert(FP64, "the Venkatakrishnan limiter is FP64 only");
          const double dxd = FD == 0 ? dx[0] : (FD == 1 ? dx[1] : dx[2]);
          const double kd = 0.3 * dxd;
          const double eps2 = kd * kd * kd;
#pragma unroll
          for (int v = 0; v < NW; ++v) {
            const int ov = orig_index_rt<MHD, NDIR>(v, FD);
            double q[4];
#pragma unroll
            for (int o = 0; o < 4; ++o) q[o] = smem[base[o] + ov * strd[o]];
            wLp[v] = q[1] + 0.25 * (q[2] - q[0]) * venk_phi(q[0], q[1], q[2], eps2);
            wRp[v] = q[2] - 0.25 * (q[3] - q[1]) * venk_phi(q[1], q[2], q[3], eps2);
          }
        } else {
#pragma unroll
          for (int v = 0; v < NW; ++v) {
            const int ov = orig_index_rt<MHD, NDIR>(v, FD);
            TF q[4];
#pragma unroll
            for (int o = 0; o < 4; ++o) q[o] = smem[base[o] + ov * strd[o]];
            const TF d0 = q[1] - q[0], d1 = q[2] - q[1], d2 = q[3] - q[2];
            TF ldw, rdw;
            face_slopes<TF, LIM, FASTF>(P.limiter, d0, d1, d2, rd, ldw, rdw);
            wLp[v] = q[1] + TF(0.5) * ldw;
            wRp[v] = q[2] - TF(0.5) * rdw;
          }
        }
        // mixed form with fix_small_values: a state near a floor goes to the
        // FP64 recomputation (its flux is marked non-finite)
        bool near = false;
        if constexpr (!FP64 && HW == 2) {
          if (P.fix_small_values) {
            TF srho = TF(0), sp = TF(0);
#pragma unroll
            for (int o = 0; o < 4; ++o) {
              srho = fmaxf(srho, fabsf(smem[base[o] + V::RHO * strd[o]]));
              sp = fmaxf(sp, fabsf(smem[base[o] + V::E * strd[o]]));
            }
            near = sv_near_floor<MHD, NDIR, GLM>(wLp, wRp, srho, sp, P);
          }
        }
        TF Fr[NW];
        // the MP5 / WENO branches of reconstruct_LR have no small-value fix of
        // the states
        stb |= face_from_states<TF, MHD, NDIR, GLM, NDIM, SOLVER, BS, FASTF>(wLp, wRp, P, TF(cg), Fr,
                                                                              HW == 2 && LIM != LIM_WENO3 && !near);
        if constexpr (RETRY) {
          // one test on the sum: an infinite or NaN flux component makes it
          // non-finite (a finite sum that overflows only costs a retry)
          TF fsum = Fr[0];
#pragma unroll
          for (int v = 1; v < NW; ++v) fsum = fsum + Fr[v];
          const bool finite = !near && isfinite(fsum);
          if (!finite) {
            s_retry = 1;
            Fr[0] = TF(NAN);
          }
        }
        // FP64: the scaled flux fC = -qdt/dx * f as in the reference; mixed:
        // the FP32 flux, scaled in FP64 by the accumulating cell thread
        const double sc = FD == 0 ? dxinv[0] : (FD == 1 ? dxinv[1] : dxinv[2]);
#pragma unroll
        for (int v = 0; v < NW; ++v) {
          const int ov = orig_index_rt<MHD, NDIR>(v, FD);
          if constexpr (FP64) flux_ref(f, FD, fl, ov) = sc * Fr[v];
          else flux_ref(f, FD, fl, ov) = Fr[v];
        }
        if (amr_mask) capture(FD, fi, fj, Fr, sc);
      }
      __syncthreads();
      if constexpr (RETRY) {
        // fix-up pass: the faces whose flux is not finite (an FP32 face of the
        // mixed form, or an FP64 face that met a special operand in the
        // unguarded arithmetic), recomputed in FP64 with the guarded forms
        if (s_retry) {
          for (int f = t; f < nface; f += THREADS) {
            int FD, fl;
            face_dir(f, FD, fl);
            bool finite = true;
            for (int v = 0; v < NW; ++v) finite = finite && isfinite(flux_ref(f, FD, fl, v));
            if (finite) continue;
            const double sc = FD == 0 ? dxinv[0] : (FD == 1 ? dxinv[1] : dxinv[2]);
            int fi, fj, base[H2], strd[H2];
            face_at(FD, fl, fi, fj, base, strd);
            const double rdd = FD == 0 ? rdel[0] : (FD == 1 ? rdel[1] : rdel[2]);
            FaceFlux64<NW> r;
            if constexpr (FP64)
              r = face_retry_fp64<TF, MHD, NDIR, GLM, NDIM, SOLVER, LIM, BS>(
                  smem, FD, base[0], base[1], base[2], base[3], strd[0], strd[1], strd[2], strd[3], rdd, cg, P);
            else  // the R cell of the face, block-local
              r = face_retry_state<MHD, NDIR, GLM, NDIM, SOLVER, LIM, BS, BN>(
                  &A, b, FD, ti0 + fi, tj0 + fj, FD == 2 ? k + 1 : k, rdd, cg);
            stb |= r.st;
            TF Fr[NW];
            for (int v = 0; v < NW; ++v) {
              Fr[v] = TF(r.F[v]);
              // FP64 keeps the scaled flux fC = -qdt/dx f, mixed the FP32 flux
              flux_ref(f, FD, fl, orig_index_rt<MHD, NDIR>(v, FD)) = FP64 ? TF(sc * r.F[v]) : Fr[v];
            }
            if (amr_mask) capture(FD, fi, fj, Fr, sc);
          }
          __syncthreads();
          if (t == 0) s_retry = 0;
        }
      }
      if (cell_thread) {
        const double sc = FP64 ? 1.0 : (D == 0 ? dxinv[0] : (D == 1 ? dxinv[1] : dxinv[2]));
        if (D == 0) {
          const int f = cj * (TB + 1) + ci;
#pragma unroll
          for (int v = 0; v < NW; ++v) {
            if constexpr (FP64) acc[v] = acc[v] + tv.fb[v * FB + f + 1] - tv.fb[v * FB + f];
            else acc[v] = acc[v] + sc * double(tv.fb[v * FB + f + 1]) - sc * double(tv.fb[v * FB + f]);
          }
        } else if (D == 1) {
          const int f = cj * TB + ci;
#pragma unroll
          for (int v = 0; v < NW; ++v) {
            // the face above the top row was computed in the x phase
            const TF up = (merge_yx && cj == TB - 1) ? tv.yx[v * TB + ci] : tv.fb[v * FB + f + TB];
            if constexpr (FP64) acc[v] = acc[v] + up - tv.fb[v * FB + f];
            else acc[v] = acc[v] + sc * double(up) - sc * double(tv.fb[v * FB + f]);
          }
        } else if constexpr (NDIM == 3) {
#pragma unroll
          for (int v = 0; v < NW; ++v) {
            const double fz = FP64 ? double(tv.fb[v * FB + t]) : sc * double(tv.fb[v * FB + t]);
            if (update) acc[v] = acc[v] + fz - fz_prev[v];
            fz_prev[v] = fz;
          }
        }
      }
      // plane k+2 ready for the z phase, ordered by the barrier below
      if (pend && D == 1) finish_async();
      // the next phase overwrites the face buffer; after the last phase the
      // barrier at the end of the plane orders the reads against the next
      // plane's writes
      if (D < NDIM - 1) __syncthreads();
    }
    // no z phase this iteration: the plane is needed by the next one (the
    // barrier at the end of the iteration orders it)
    if (pend) finish_async();
    }  // face phases
    if (update && cell_thread) {
      // ---- small values on wnew (src/mod_finite_volume.t:326-333; the
      // Hancock predictor checks after the sources instead)
      if (SOLVER != SOLVER_HANCOCK && P.fix_small_values) {
        if (small_values<double, MHD, NDIR, GLM>(acc, false, P) && P.small_values_method != 1) stb |= ST_SMALL_VALUE;
      }
      // ---- unsplit divB sources (addsource2 -> mhd_add_source)
      if constexpr (MHD) {
        if (NDIM > 1) {
          // addsource2 with qdt (idimmax - idimmin + 1) / ndim
          const double qsrc = qdt * double(dsel < 0 ? NDIM : 1) / double(NDIM);
          if constexpr (GLM) {
            // add_source_glm (src/mhd/mod_mhd_phys.t:5472-5531)
            double mindx = dx[0];
#pragma unroll
            for (int d = 1; d < NDIM; ++d) mindx = fmin(mindx, dx[d]);
            if (P.glm_alpha < 0.0) {
              acc[V::PSI] = fabs(P.glm_alpha) * A.uin[cell_offset<NDIM>(b, NW, V::PSI, bi, bj, k, BN)];
            } else {
              acc[V::PSI] = exp(-(qsrc * cg * P.glm_alpha) / mindx) * acc[V::PSI];
            }
            if (P.glm_extended) {
              auto nbv = [&](int d, int s, int v) -> double {  // wCT at cell +/- e_d
                if (d == 0) return double(tv.at(slot, v, ci + s, cj));
                if (d == 1) return double(tv.at(slot, v, ci, cj + s));
                return double(tv.ring[(ring_slot<HW>(k + s) * NW + v) * (TB * TB) + cj * TB + ci]);
              };
#pragma unroll
              for (int d = 0; d < NDIM; ++d) {
                const double g = ((nbv(d, 1, V::PSI) - nbv(d, -1, V::PSI)) * 0.5) / dx[d];
                acc[V::E] = acc[V::E] - qsrc * double(tv.at(slot, V::B0 + d, ci, cj)) * g;
              }
              double divb = 0.0;
#pragma unroll
              for (int d = 0; d < NDIM; ++d)
                divb = divb + 0.5 * (nbv(d, 1, V::B0 + d) - nbv(d, -1, V::B0 + d)) * (1.0 / dx[d]);
#pragma unroll
              for (int c = 0; c < NDIR; ++c)
                acc[V::M0 + c] = acc[V::M0 + c] - qsrc * double(tv.at(slot, V::B0 + c, ci, cj)) * divb;
            }
          } else if (P.divb == DIVB_LINDE) {
            // the reference leaves out the cell layer next to a level-jump
            // face "for AMR stability" (src/mhd/mod_mhd_phys.t:5616-5642)
            const bool jump_layer = amr_mask && (((amr_mask & 1) && bi == 0) || ((amr_mask & 2) && bi == BN - 1) ||
                                                 ((amr_mask & 4) && bj == 0) || ((amr_mask & 8) && bj == BN - 1));
            if constexpr (NDIM == 2) if (!jump_layer) {
              // add_source_linde (src/mhd/mod_mhd_phys.t:5599-5665)
              auto divb_at = [&](int i, int j) -> double {
                double d = 0.5 * (double(tv.at(slot, V::B0, i + 1, j)) - double(tv.at(slot, V::B0, i - 1, j))) * (1.0 / dx[0]);
                d = d + 0.5 * (double(tv.at(slot, V::B0 + 1, i, j + 1)) - double(tv.at(slot, V::B0 + 1, i, j - 1))) * (1.0 / dx[1]);
                return d;
              };
              const double inv2 = 1.0 / (dx[0] * dx[0]) + 1.0 / (dx[1] * dx[1]);
#pragma unroll
              for (int d = 0; d < 2; ++d) {
                const double dp = d == 0 ? divb_at(ci + 1, cj) : divb_at(ci, cj + 1);
                const double dm = d == 0 ? divb_at(ci - 1, cj) : divb_at(ci, cj - 1);
                double g = (dp - dm) * 0.5;
                g = g / dx[d];
                g = g * P.divbdiff / inv2;
                acc[V::B0 + d] = acc[V::B0 + d] + g;
                acc[V::E] = acc[V::E] + double(tv.at(slot, V::B0 + d, ci, cj)) * g;
              }
            }
          }
          if (P.fix_small_values) {
            if (small_values<double, MHD, NDIR, GLM>(acc, false, P) && P.small_values_method != 1) stb |= ST_SMALL_VALUE;
          }
        }
      }
      // ---- 'exit hancock' small-value check (src/mod_finite_volume.t:106-109)
      if (SOLVER == SOLVER_HANCOCK && P.fix_small_values) {
        if (small_values<double, MHD, NDIR, GLM>(acc, false, P) && P.small_values_method != 1) stb |= ST_SMALL_VALUE;
      }
      if (!isfinite(acc[V::RHO]) || !isfinite(acc[V::E])) stb |= ST_NAN;
#pragma unroll
      for (int v = 0; v < NW; ++v) A.uout[cell_offset<NDIM>(b, NW, v, bi, bj, k, BN)] = acc[v];
    }
    // the next iteration (or the next block) overwrites ring slot (k-1)&3
    // and the halo strips, which the sources above read
    __syncthreads();
  }
  // the reference restores the whole block to wCT on a small-value crash
  // (finite_volume; hancock does not).  With 'average' a small value sends
  // the block to the whole-block recomputation instead (smallavg.cu), and a
  // non-finite result goes to the block's status: the recomputation reports
  // it only for the blocks it does not replace (another thread or CTA of
  // the block may be the one that saw the small value).
  if (P.small_values_method == 2) {
    if (stb & (ST_SMALL_VALUE | ST_NAN))
      atomicOr(A.block_status + b, ((stb & ST_SMALL_VALUE) ? ST_SV_AVG : 0u) | (stb & ST_NAN));
    stb &= ~(ST_SMALL_VALUE | ST_NAN);
  } else if (SOLVER != SOLVER_HANCOCK && (stb & ST_SMALL_VALUE)) {
    atomicOr(A.block_status + b, ST_SMALL_VALUE);
  }
  st |= stb;
  }  // while (g < gend)
  if (st) atomicOr(A.status, st);
}

}  // namespace amrvac
