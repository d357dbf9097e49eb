// Kernel launchers shared by the per-physics translation units.
#pragma once

#include <cuda_runtime.h>

#include "stage.cuh"

namespace amrvac {

// ---------------------------------------------------------------- getdt
// getdt_courant (src/mod_dt.t:160-287) per block, reduced over all blocks.
// red[0] <- max over blocks of the block's courant sum (maxsum: max_cells
// sum_d cmax_d/dx_d; summax / minimum per the reference), red[1] <- max cmax.
struct GetdtArgs {
  const double *u;
  const double *dxb;
  int nblocks;
  int bn;  // block edge
  int type_courant;
  unsigned long long *red;
  PhysParams P;
  uint32_t *status;  // the context's status word: the small-value check of getdt
  const uint32_t *skip;  // 'average': blocks flagged ST_SV_AVG are reduced by sv_getdt_kernel
};

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Non-negative doubles order like their bit patterns.
__device__ __forceinline__ void atomic_max_pos(unsigned long long *a, double v) {
  if (v > 0.0) atomicMax(a, (unsigned long long)__double_as_longlong(v));
}

template <bool MHD, int NDIR, bool GLM, int NDIM>
__global__ void __launch_bounds__(256) getdt_kernel(const GetdtArgs A) {
  using V = Vars<MHD, NDIR, GLM>;
  constexpr int NW = V::NW;
  const int bn = A.bn;
  const int ncell = bn * (NDIM >= 2 ? bn : 1) * (NDIM == 3 ? bn : 1);
  const int b = blockIdx.x;
  const int t = threadIdx.x;
  if (A.skip && (A.skip[b] & ST_SV_AVG)) return;
  double dxinv[3];
#pragma unroll
  for (int d = 0; d < NDIM; ++d) dxinv[d] = 1.0 / A.dxb[b * 3 + d];
  double mtot = 0.0, mcm = 0.0, mdim[3] = {0.0, 0.0, 0.0};
  // the block's cells, x fastest (coalesced), 256 at a time; c is the
  // cell's index within its block-variable row (cell_offset's layout)
  const double *ub = A.u + (size_t)b * NW * ncell;
#pragma unroll 2
  for (int c = t; c < ncell; c += 256) {
    double w[NW];
#pragma unroll
    for (int v = 0; v < NW; ++v) w[v] = __ldg(ub + (size_t)v * ncell + c);
    // getdt_courant takes the primitives through phys_to_primitive, small-value
    // fix included (src/mod_dt.t:189-191)
    if (A.P.fix_small_values) {
      if (small_values<double, MHD, NDIR, GLM>(w, false, A.P) && A.P.small_values_method != 1 && A.status)
        atomicOr(A.status, ST_SMALL_VALUE);
    }
    to_primitive<MHD, NDIR, GLM>(w, A.P);
    double tot = 0.0;
#pragma unroll
    for (int d = 0; d < NDIM; ++d) {
      double cm;
      if constexpr (MHD) {
        double cf;
        if (d == 0) cf = fast_speed<double, NDIR, V::B0 + 0>(w, A.P);
        else if (d == 1) cf = fast_speed<double, NDIR, V::B0 + (NDIR > 1 ? 1 : 0)>(w, A.P);
        else cf = fast_speed<double, NDIR, V::B0 + (NDIR > 2 ? 2 : 0)>(w, A.P);
        cm = fabs(w[V::M0 + d]) + cf;
      } else {
        cm = fabs(w[V::M0 + d]) + sqrt(A.P.gamma * w[V::E] / w[V::RHO]);
      }
      const double c = cm * dxinv[d];
      tot = d == 0 ? c : tot + c;
      mdim[d] = fmax(mdim[d], c);
      mcm = fmax(mcm, cm);
    }
    mtot = fmax(mtot, tot);
  }
  __shared__ double red[4][8];
  const int lane = t & 31, wid = t >> 5;
  double r0 = warp_max(mtot), r1 = warp_max(mcm);
  double r2[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) r2[d] = warp_max(mdim[d]);
  if (lane == 0) {
    red[0][wid] = r0; red[1][wid] = r1;
    red[2][wid] = r2[0]; red[3][wid] = r2[1];
  }
  __shared__ double red3[8];
  if (lane == 0) red3[wid] = r2[2];
  __syncthreads();
  if (t == 0) {
    double a0 = 0, a1 = 0, d0 = 0, d1 = 0, d2 = 0;
    for (int q = 0; q < 8; ++q) {
      a0 = fmax(a0, red[0][q]); a1 = fmax(a1, red[1][q]);
      d0 = fmax(d0, red[2][q]); d1 = fmax(d1, red[3][q]); d2 = fmax(d2, red3[q]);
    }
    double x;
    if (A.type_courant == 1) {
      x = a0;
    } else {
      double dd[3] = {d0, d1, d2};
      double courantmax = 0.0, tot = 0.0;
      for (int d = 0; d < NDIM; ++d) {
        courantmax = fmax(courantmax, dd[d]);
        tot = tot + courantmax;
      }
      x = A.type_courant == 2 ? tot : courantmax;
    }
    atomic_max_pos(A.red + 0, x);
    atomic_max_pos(A.red + 1, a1);
  }
}

// ---------------------------------------------------------------- points
struct PointArgs {
  int n;
  const double *a, *b, *c, *d;  // inputs (state-major [n][nw])
  double *out, *out2;
  double cg;
  PhysParams P;
};

template <bool MHD, int NDIR, bool GLM, int NDIM, int SOLVER, int D>
__global__ void riemann_points_kernel(const PointArgs A) {
  using V = Vars<MHD, NDIR, GLM>;
  constexpr int NW = V::NW;
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= A.n) return;
  double wL[NW], wR[NW], F[NW];
#pragma unroll
  for (int v = 0; v < NW; ++v) {
    const int ov = orig_index<MHD, NDIR, D>(v);
    wL[v] = A.a[(size_t)p * NW + ov];
    wR[v] = A.b[(size_t)p * NW + ov];
  }
  face_from_states<double, MHD, NDIR, GLM, NDIM, SOLVER, 0>(wL, wR, A.P, A.cg, F);
#pragma unroll
  for (int v = 0; v < NW; ++v) A.out[(size_t)p * NW + orig_index<MHD, NDIR, D>(v)] = F[v];
}

template <bool MHD, int NDIR, bool GLM, int D>
__global__ void flux_points_kernel(const PointArgs A) {
  using V = Vars<MHD, NDIR, GLM>;
  constexpr int NW = V::NW;
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= A.n) return;
  double wc[NW], w[NW], f[NW];
#pragma unroll
  for (int v = 0; v < NW; ++v) { wc[v] = A.a[(size_t)p * NW + v]; w[v] = A.b[(size_t)p * NW + v]; }
  phys_flux<double, MHD, NDIR, GLM, D>(wc, w, A.cg, f);
#pragma unroll
  for (int v = 0; v < NW; ++v) A.out[(size_t)p * NW + v] = f[v];
}

template <bool MHD, int NDIR, bool GLM, int D>
__global__ void cbounds_points_kernel(const PointArgs A) {
  using V = Vars<MHD, NDIR, GLM>;
  constexpr int NW = V::NW;
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= A.n) return;
  double lc[NW], rc[NW], lp[NW], rp[NW];
#pragma unroll
  for (int v = 0; v < NW; ++v) {
    lc[v] = A.a[(size_t)p * NW + v]; rc[v] = A.b[(size_t)p * NW + v];
    lp[v] = A.c[(size_t)p * NW + v]; rp[v] = A.d[(size_t)p * NW + v];
  }
  double cmax, cmin = 0.0;
  if (A.out2) cbounds<double, MHD, NDIR, GLM, D, true>(lc, rc, lp, rp, A.P, cmax, cmin);
  else cbounds<double, MHD, NDIR, GLM, D, false>(lc, rc, lp, rp, A.P, cmax, cmin);
  A.out[p] = cmax;
  if (A.out2) A.out2[p] = cmin;
}

// ---------------------------------------------------------------- a2max
// phys_get_a2max (hd_get_a2max src/hd/mod_hd_phys.t:813-833; MHD the same,
// src/mhd/mod_mhd_phys.t:2678-2698) reduced as getdt_courant and setdt do
// for schmid1 (src/mod_dt.t:193-197, 130): per block and direction d the
// maximum over its cells and conserved variables of
// |-w(i+2) + 16 w(i+1) - 30 w(i) + 16 w(i-1) - w(i-2)|, / 12 / dx_d^2, then
// the maximum over blocks into out[d].  One CTA per z-plane of a block.
template <int NW, int NDIM, int BN = BN16>
__global__ void __launch_bounds__(256) a2max_kernel(const StageArgs A, double *out) {
  constexpr int PL = NDIM == 3 ? BN : 1;
  const int b = blockIdx.x / PL, k = blockIdx.x - (blockIdx.x / PL) * PL;
  auto w = [&](int ii, int jj, int kk, int v) {
    uint32_t flip;
    const int blk = resolve_cell<NDIM>(A, b, ii, jj, kk, flip, BN);
    const double x = blk >= 0 ? __ldg(A.uin + cell_offset<NDIM>(blk, NW, v, ii, jj, kk, BN))
                              : __ldg(A.gbuf + ghost_offset<NDIM>(-2 - blk, NW, v, ii, jj, kk, BN));
    return ((flip >> v) & 1u) ? -x : x;
  };
  __shared__ double red[8];
#pragma unroll 1
  for (int d = 0; d < NDIM; ++d) {
    const int e0 = d == 0, e1 = d == 1, e2 = d == 2;
    double m = 0.0;
    for (int c = threadIdx.x; c < BN * BN; c += 256) {  // the cells of the plane
      const int i = c % BN, j = c / BN;
#pragma unroll
      for (int v = 0; v < NW; ++v) {
        const double a = fabs(((((-w(i + 2 * e0, j + 2 * e1, k + 2 * e2, v) + 16.0 * w(i + e0, j + e1, k + e2, v)) -
                                 30.0 * w(i, j, k, v)) +
                                16.0 * w(i - e0, j - e1, k - e2, v)) -
                               w(i - 2 * e0, j - 2 * e1, k - 2 * e2, v)));
        m = fmax(m, a);
      }
    }
    m = warp_max(m);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
      double mm = red[0];
      for (int q = 1; q < 8; ++q) mm = fmax(mm, red[q]);
      const double dx = A.dxb[b * 3 + d];
      atomic_max_pos(reinterpret_cast<unsigned long long *>(out + d), mm / 12.0 / (dx * dx));
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------- Linde, 3-D
// add_source_linde (src/mhd/mod_mhd_phys.t:5599-5665) for 3-D blocks, run
// after the stage kernel on its output: w(B_d) += g_d, w(e) += wCT(B_d) g_d
// with g_d = divbdiff / sum_d(1/dx_d^2) * d(divB)/dx_d (central), divB of wCT
// (central, get_divb with mhd_divb_nth = 1), leaving out the cell layers next
// to level-jump faces; then the small-value check of mhd_add_source.  Its
// stencil (divB at the six neighbours: B two cells out and across the z
// planes' halos) is gathered here through the stage's neighbour resolution
// (and the level-jump ghost buffers); one CTA per z-plane of a block.
template <int NDIR, int BN = BN16>
__global__ void __launch_bounds__(256) linde3d_kernel(const StageArgs A) {
  using V = Vars<true, NDIR, false>;
  constexpr int NW = V::NW;
  const int b = blockIdx.x / BN, k = blockIdx.x - (blockIdx.x / BN) * BN;
  if (b >= A.nblocks) return;
  const int m = A.amr_face ? A.amr_face[b] : 0;
  for (int c = threadIdx.x; c < BN * BN; c += 256) {  // the cells of the plane
  const int i = c % BN, j = c / BN;
  if (m && (((m & 1) && i == 0) || ((m & 2) && i == BN - 1) || ((m & 4) && j == 0) || ((m & 8) && j == BN - 1) ||
            ((m & 16) && k == 0) || ((m & 32) && k == BN - 1)))
    continue;
  double dx[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) dx[d] = A.dxb[b * 3 + d];
  auto bct = [&](int ii, int jj, int kk, int c) -> double {  // wCT's B_c, up to two cells outside
    uint32_t flip;
    const int blk = resolve_cell<3>(A, b, ii, jj, kk, flip, BN);
    const int v = V::B0 + c;
    const double x = blk >= 0 ? __ldg(A.uin + cell_offset<3>(blk, NW, v, ii, jj, kk, BN))
                              : __ldg(A.gbuf + ghost_offset<3>(-2 - blk, NW, v, ii, jj, kk, BN));
    return ((flip >> v) & 1u) ? -x : x;
  };
  auto divb = [&](int ii, int jj, int kk) {
    double d = 0.5 * (bct(ii + 1, jj, kk, 0) - bct(ii - 1, jj, kk, 0)) * (1.0 / dx[0]);
    d = d + 0.5 * (bct(ii, jj + 1, kk, 1) - bct(ii, jj - 1, kk, 1)) * (1.0 / dx[1]);
    d = d + 0.5 * (bct(ii, jj, kk + 1, 2) - bct(ii, jj, kk - 1, 2)) * (1.0 / dx[2]);
    return d;
  };
  const double inv2 = (1.0 / (dx[0] * dx[0]) + 1.0 / (dx[1] * dx[1])) + 1.0 / (dx[2] * dx[2]);
  double w[NW];
#pragma unroll
  for (int v = 0; v < NW; ++v) w[v] = A.uout[cell_offset<3>(b, NW, v, i, j, k, BN)];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double dp = d == 0 ? divb(i + 1, j, k) : (d == 1 ? divb(i, j + 1, k) : divb(i, j, k + 1));
    const double dm = d == 0 ? divb(i - 1, j, k) : (d == 1 ? divb(i, j - 1, k) : divb(i, j, k - 1));
    double g = (dp - dm) * 0.5;
    g = g / dx[d];
    g = g * A.P.divbdiff / inv2;
    w[V::B0 + d] = w[V::B0 + d] + g;
    w[V::E] = w[V::E] + __ldg(A.uin + cell_offset<3>(b, NW, V::B0 + d, i, j, k, BN)) * g;
  }
  if (A.P.fix_small_values) {
    if (small_values<double, true, NDIR, false>(w, false, A.P) && A.P.small_values_method != 1)
      atomicOr(A.status, ST_SMALL_VALUE);
  }
#pragma unroll
  for (int v = 0; v < NW; ++v) A.uout[cell_offset<3>(b, NW, v, i, j, k, BN)] = w[v];
  }  // cells of the plane
}

// ---------------------------------------------------------------- dispatch
struct KernelSet {
  cudaError_t (*prepare)() = nullptr;
  int (*ctas_per_sm)() = nullptr;
  cudaError_t (*stage)(const StageArgs &, int nctas, cudaStream_t) = nullptr;
  // MUSCL-Hancock predictor of twostep Predictor_Corrector (tvdlf sets only)
  cudaError_t (*hancock)(const StageArgs &, int nctas, cudaStream_t) = nullptr;
  // the 3-D Linde divB source after a stage (3-D MHD sets without GLM)
  cudaError_t (*linde3d)(const StageArgs &, cudaStream_t) = nullptr;
  // a2max_global of schmid1 (every set)
  cudaError_t (*a2max)(const StageArgs &, double *out, cudaStream_t) = nullptr;
  cudaError_t (*getdt)(const GetdtArgs &, cudaStream_t) = nullptr;
  cudaError_t (*riemann_points)(const PointArgs &, int idim, cudaStream_t) = nullptr;
  cudaError_t (*flux_points)(const PointArgs &, int idim, cudaStream_t) = nullptr;
  cudaError_t (*cbounds_points)(const PointArgs &, int idim, cudaStream_t) = nullptr;
  size_t stage_smem = 0;
  int bn = BN16;  // the block edge the stage kernels were built for
  // Stage-kernel variants the autotuner times (variant 0 is `stage`): per
  // variant the launch, its occupancy query, threads per CTA, the CTAs per
  // SM its registers are capped for, and asynchronous plane staging.
  static constexpr int MAXVAR = 4;
  int nvar = 1;
  cudaError_t (*stage_v[MAXVAR])(const StageArgs &, int nctas, cudaStream_t) = {};
  int (*ctas_v[MAXVAR])() = {};
  cudaError_t (*prepare_v[MAXVAR])() = {};
  int var_threads[MAXVAR] = {}, var_minb[MAXVAR] = {}, var_async[MAXVAR] = {};
};

// One stage-kernel variant of a scheme (see stage_variant).
template <bool MHD, int NDIR, bool GLM, int NDIM, int SOLVER, int LIM, int BS, class TF, int BN, int VAR>
struct StageVar {
  using V = Vars<MHD, NDIR, GLM>;
  using O = StageOcc<TF, LIM, BN, VAR>;
  static constexpr size_t SMEM = Tile<TF, V::NW, NDIM, HaloW<LIM>::value, tile_edge(BN)>::BYTES;
  static cudaError_t prepare() {
    return cudaFuncSetAttribute(fv_stage_kernel<TF, MHD, NDIR, GLM, NDIM, SOLVER, LIM, BS, BN, VAR>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM);
  }
  static cudaError_t stage(const StageArgs &A, int nctas, cudaStream_t s) {
    fv_stage_kernel<TF, MHD, NDIR, GLM, NDIM, SOLVER, LIM, BS, BN, VAR><<<nctas, O::THREADS, SMEM, s>>>(A);
    return cudaGetLastError();
  }
  static int ctas_per_sm() {
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &n, fv_stage_kernel<TF, MHD, NDIR, GLM, NDIM, SOLVER, LIM, BS, BN, VAR>, O::THREADS, SMEM) != cudaSuccess)
      return 1;
    return n > 0 ? n : 1;
  }
  static void add(KernelSet &k, int slot) {
    k.stage_v[slot] = &stage;
    k.ctas_v[slot] = &ctas_per_sm;
    k.prepare_v[slot] = &prepare;
    k.var_threads[slot] = O::THREADS;
    k.var_minb[slot] = O::MINB;
    k.var_async[slot] = O::ASYNC && sizeof(TF) == 8 && NDIM == 3 && tile_edge(BN) == BN && HaloW<LIM>::value == 2;
    if (slot + 1 > k.nvar) k.nvar = slot + 1;
  }
};

template <bool MHD, int NDIR, bool GLM, int NDIM, int SOLVER, int LIM = 0, int BS = 0, class TF = double,
          int BN = BN16>
struct Launch {
  using V = Vars<MHD, NDIR, GLM>;
  static constexpr int THREADS = StageOcc<TF, LIM, BN>::THREADS;
  static constexpr size_t SMEM = Tile<TF, V::NW, NDIM, HaloW<LIM>::value, tile_edge(BN)>::BYTES;
  // typepred1 = fs_hancock for tvdlf and tvdmu (src/io/mod_input_output.t:787-797)
  static constexpr bool HAS_HANCOCK = (SOLVER == SOLVER_TVDLF || SOLVER == SOLVER_TVDMU) && sizeof(TF) == 8;
  static cudaError_t prepare() {
    cudaError_t e = cudaFuncSetAttribute(fv_stage_kernel<TF, MHD, NDIR, GLM, NDIM, SOLVER, LIM, BS, BN>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM);
    if constexpr (HAS_HANCOCK) {
      if (e == cudaSuccess)
        e = cudaFuncSetAttribute(fv_stage_kernel<TF, MHD, NDIR, GLM, NDIM, SOLVER_HANCOCK, LIM, BS, BN>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM);
    }
    return e;
  }
  static cudaError_t stage(const StageArgs &A, int nctas, cudaStream_t s) {
    fv_stage_kernel<TF, MHD, NDIR, GLM, NDIM, SOLVER, LIM, BS, BN><<<nctas, THREADS, SMEM, s>>>(A);
    return cudaGetLastError();
  }
  static cudaError_t a2max(const StageArgs &A, double *out, cudaStream_t s) {
    a2max_kernel<V::NW, NDIM, BN><<<A.nblocks * (NDIM == 3 ? BN : 1), 256, 0, s>>>(A, out);
    return cudaGetLastError();
  }
  static cudaError_t linde3d(const StageArgs &A, cudaStream_t s) {
    if constexpr (MHD && NDIM == 3 && !GLM) {
      linde3d_kernel<NDIR, BN><<<A.nblocks * BN, 256, 0, s>>>(A);
      return cudaGetLastError();
    } else {
      return cudaErrorNotSupported;
    }
  }
  static cudaError_t hancock(const StageArgs &A, int nctas, cudaStream_t s) {
    if constexpr (HAS_HANCOCK) {
      fv_stage_kernel<TF, MHD, NDIR, GLM, NDIM, SOLVER_HANCOCK, LIM, BS, BN><<<nctas, THREADS, SMEM, s>>>(A);
      return cudaGetLastError();
    } else {
      return cudaErrorNotSupported;
    }
  }
  static int ctas_per_sm() {
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &n, fv_stage_kernel<TF, MHD, NDIR, GLM, NDIM, SOLVER, LIM, BS, BN>, THREADS, SMEM) != cudaSuccess)
      return 1;
    return n > 0 ? n : 1;
  }
  static cudaError_t getdt(const GetdtArgs &A, cudaStream_t s) {
    getdt_kernel<MHD, NDIR, GLM, NDIM><<<A.nblocks, 256, 0, s>>>(A);
    return cudaGetLastError();
  }
  template <int D>
  static void rp(const PointArgs &A, cudaStream_t s) {
    riemann_points_kernel<MHD, NDIR, GLM, NDIM, SOLVER, D><<<(A.n + 127) / 128, 128, 0, s>>>(A);
  }
  static cudaError_t riemann_points(const PointArgs &A, int idim, cudaStream_t s) {
    if (idim == 1) rp<0>(A, s);
    else if (idim == 2 && NDIM >= 2) rp<NDIM >= 2 ? 1 : 0>(A, s);
    else if (idim == 3 && NDIM >= 3) rp<NDIM >= 3 ? 2 : 0>(A, s);
    else return cudaErrorInvalidValue;
    return cudaGetLastError();
  }
  template <int D>
  static void fp(const PointArgs &A, cudaStream_t s) {
    flux_points_kernel<MHD, NDIR, GLM, D><<<(A.n + 127) / 128, 128, 0, s>>>(A);
  }
  static cudaError_t flux_points(const PointArgs &A, int idim, cudaStream_t s) {
    if (idim == 1) fp<0>(A, s);
    else if (idim == 2 && NDIR >= 2) fp<NDIR >= 2 ? 1 : 0>(A, s);
    else if (idim == 3 && NDIR >= 3) fp<NDIR >= 3 ? 2 : 0>(A, s);
    else return cudaErrorInvalidValue;
    return cudaGetLastError();
  }
  template <int D>
  static void cp(const PointArgs &A, cudaStream_t s) {
    cbounds_points_kernel<MHD, NDIR, GLM, D><<<(A.n + 127) / 128, 128, 0, s>>>(A);
  }
  static cudaError_t cbounds_points(const PointArgs &A, int idim, cudaStream_t s) {
    if (idim == 1) cp<0>(A, s);
    else if (idim == 2 && NDIR >= 2) cp<NDIR >= 2 ? 1 : 0>(A, s);
    else if (idim == 3 && NDIR >= 3) cp<NDIR >= 3 ? 2 : 0>(A, s);
    else return cudaErrorInvalidValue;
    return cudaGetLastError();
  }
  static KernelSet set() {
    KernelSet k;
    k.prepare = &prepare;
    k.ctas_per_sm = &ctas_per_sm;
    k.stage = &stage;
    if (HAS_HANCOCK) k.hancock = &hancock;
    if (MHD && NDIM == 3 && !GLM) k.linde3d = &linde3d;
    k.a2max = &a2max;
    k.getdt = &getdt;
    k.riemann_points = &riemann_points;
    k.flux_points = &flux_points;
    k.cbounds_points = &cbounds_points;
    k.stage_smem = SMEM;
    k.bn = BN;
    StageVar<MHD, NDIR, GLM, NDIM, SOLVER, LIM, BS, TF, BN, 0>::add(k, 0);
    return k;
  }
};

// Lookup key for one physics / dimension / solver combination.
struct KernelKey {
  bool mhd;
  int ndim, ndir;
  bool glm;
  int solver;
  int limiter;     // used to pick a compile-time specialised stage kernel
  int boundspeed;
  bool mixed;      // FP32 face arithmetic (mixed form)
  int bn;          // block edge (block_nx)
};

bool lookup_hd(const KernelKey &k, KernelSet *out);
// small_values_method 'average' (smallavg.cu): detection, whole-block stage
// and getdt of the flagged blocks; scratch per CTA (SvScratch).
struct SvScratch;
struct SvSet {
  cudaError_t (*detect)(const StageArgs &, const double *reg, cudaStream_t) = nullptr;
  cudaError_t (*stage)(const StageArgs &, const double *snap_base, const double *snap_in, SvScratch, int nctas,
                       cudaStream_t) = nullptr;
  cudaError_t (*getdt)(const StageArgs &, const double *reg, int type_courant, unsigned long long *red, SvScratch,
                       int nctas, cudaStream_t) = nullptr;
};
struct SvScratch {
  double *base;
  size_t per_cta;  // doubles per CTA
};
bool lookup_sv(const KernelKey &k, SvSet *out);
// The variants 1..3 of the benchmark schemes' stage kernels (k_tune.cu).
bool add_stage_variants(const KernelKey &k, KernelSet *out);
// block edges other than 16 (k_blocks.cuh, one unit per edge)
bool lookup_bn8(const KernelKey &k, KernelSet *out);
bool lookup_bn10(const KernelKey &k, KernelSet *out);
bool lookup_bn12(const KernelKey &k, KernelSet *out);
bool lookup_bn32(const KernelKey &k, KernelSet *out);
bool lookup_mp5_hd(const KernelKey &k, KernelSet *out);
bool lookup_mp5_mhd(const KernelKey &k, KernelSet *out);
bool lookup_mhd2(const KernelKey &k, KernelSet *out);
bool lookup_mhd3(const KernelKey &k, KernelSet *out);

}  // namespace amrvac
