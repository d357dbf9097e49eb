// Batched ensembles: many independent hydrodynamics runs — 1-D and 2-D, of
// uneven sizes, each with its own Riemann solver, limiter, time step and end
// time — advanced together, one persistent kernel launch per RK stage for all
// of them.  Each instance is one standalone run of the reference's time loop
// (src/amrvac.t:241-343: setdt, exit check, advance) on a uniform level-1
// grid of 16^d blocks; instances never exchange data.
//
// Device organisation.  Blocks of each dimensionality live in their own pool
// (1-D: nw = 3, 2-D: nw = 4), interior cells only, [block][var][y][x], three
// registers.  The unit of work is a tile of 16 rows x 16 cells: one 2-D block,
// or sixteen 1-D blocks packed as rows (grouped by scheme so a tile's rows
// usually share solver and limiter).  The tile list holds the 2-D tiles first,
// then the 1-D tiles; persistent CTAs stride over it.  Instances that have
// finished are dropped from the list by the host between graph chunks, and
// skipped by a flag test in the meantime.
//
// Per-instance state on the device: dt, time, time_max, dx, solver, limiter,
// done flag, step count and the getdt reduction word.  One step is
//   getdt (per-instance max of the maxsum courant number) -> finalize (dt per
//   instance, dtmin check, final_dt_reduction, exit test) -> RK stages ->
//   advance time,
// captured into a CUDA graph of several steps.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/amrvac_gpu.h"
#include "aux.cuh"
#include "kernels.cuh"

namespace amrvac {
int record_error(int code, const std::string &msg);  // capi.cu

constexpr int ENS_ROWS = 16;  // rows per tile

struct EnsArgs {
  StageArgs sa[2];           // per pool (index ndim-1): uin/ubase/uout, nbr, bc, status, P
  const int *inst[2];        // instance of every block, per pool
  const int *tiles;          // [tile][16] block ids (2-D tile: entry 0; 1-D tile: one per row, -1 empty)
  const int *ntiles;         // device: [0] 2-D tiles, [1] all tiles
  double a_base, b_in, dtfactor;
  const double *dt;          // [ninst]
  const double *dx;          // [ninst][2]
  const int *solver;         // [ninst] SOLVER_*
  const int *limiter;        // [ninst] LIM_*
  const int *done;           // [ninst]
  unsigned long long *red;   // [ninst] getdt accumulators
  uint32_t *inst_status;     // [ninst] sticky status per instance
};

struct EnsRow {
  int blk, inst, solver, limiter;
  double sc[2];   // -qdt/dx per direction
  double rd[2];   // cada3 1/(radius*dx)^2 per direction
  double dxinv[2];
};

// Fill the per-row table of a tile (threads 0..15); returns, for all
// threads, whether any row of the tile is active.
template <int ND>
__device__ __forceinline__ bool ens_rows(const EnsArgs &A, int tile, bool for_getdt, EnsRow *rows) {
  const int t = threadIdx.x;
  bool act = false;
  if (t < ENS_ROWS) {
    const int b = A.tiles[tile * ENS_ROWS + (ND == 2 ? 0 : t)];
    int in = b >= 0 ? A.inst[ND - 1][b] : -1;
    if (in >= 0 && A.done[in]) in = -1;
    EnsRow &R = rows[t];
    R.blk = b;
    R.inst = in;
    if (in >= 0) {
      R.solver = A.solver[in];
      R.limiter = A.limiter[in];
      const double qdt = for_getdt ? 0.0 : A.dtfactor * A.dt[in];
#pragma unroll
      for (int d = 0; d < ND; ++d) {
        const double dx = A.dx[in * 2 + d];
        R.sc[d] = -qdt / dx;
        const double r = A.sa[0].P.cada3_radius * dx;
        R.rd[d] = 1.0 / (r * r);
        R.dxinv[d] = 1.0 / dx;
      }
    }
    act = in >= 0;
  }
  return __syncthreads_or(act) != 0;
}

// The mixed form's FP32 faces use the hardware approximations (rcp.approx /
// sqrt.approx, about one FP32 ulp) as the stage kernel's do; FP64 faces keep
// the guarded division (this kernel has no recomputation pass).
template <class TF, int ND, int SOLVER>
__device__ __forceinline__ uint32_t ens_face(TF *wLp, TF *wRp, const PhysParams &P, TF *F) {
  return face_from_states<TF, false, ND, false, ND, SOLVER, 0, sizeof(TF) == 4>(wLp, wRp, P, TF(0), F);
}

// Stage kernel organisation: 288 threads.  Threads 0..255 own the cells of
// the tile (ci = t % 16, row cj = t / 16) and compute the x-face and the
// y-face on the low side of their cell; the ninth warp computes the 16 x-faces
// of the high side (lanes 0..15) and the 16 y-faces of the top (lanes 16..31),
// so every thread handles at most two faces.  One shared tile and a triple-
// buffered row table, so one tile costs two barriers:
//   stage cells + halos (+ row table of the next tile, by the ninth warp)
//   | barrier | all faces of both directions | barrier | accumulate + store.
constexpr int ENS_THREADS = 288;

// Shared tile of one buffer, in TF elements, for up to 4 variables.
template <class TF>
struct EnsTile {
  static constexpr int NWM = 4;
  static constexpr int TOTAL = NWM * (BN16 * BN16 + BN16 * 4 + 4 * BN16 + 2 * (BN16 + 1) * BN16);
};

template <class TF, int NW>
struct EnsView {
  TF *ring, *hx, *hy, *fbx, *fby;  // [v][j][i], [v][j][c], [v][r][i], [v][j][17], [v][17][i]
  __device__ __forceinline__ explicit EnsView(TF *s) {
    ring = s;
    hx = ring + NW * BN16 * BN16;
    hy = hx + NW * BN16 * 4;
    fbx = hy + NW * 4 * BN16;
    fby = fbx + NW * (BN16 + 1) * BN16;
  }
  // element offset of variable 0 at (i, j) in [-2, 17] x [0, 15] or [0, 15] x [-2, 17],
  // and the stride between variables
  __device__ __forceinline__ void addr(int i, int j, int &base, int &stride) const {
    const bool ii = (unsigned)i < (unsigned)BN16;
    const bool jj = (unsigned)j < (unsigned)BN16;
    if (ii && jj) { base = j * BN16 + i; stride = BN16 * BN16; }
    else if (jj) { base = NW * BN16 * BN16 + j * 4 + halo_slot_w<2>(i); stride = BN16 * 4; }
    else { base = NW * BN16 * BN16 + NW * BN16 * 4 + halo_slot_w<2>(j) * BN16 + i; stride = 4 * BN16; }
  }
};

// Row table entry of one row of a tile (2-D tile: the block, all rows alike).
__device__ __forceinline__ void ens_fill_row(const EnsArgs &A, int tile, bool two_d, int row, EnsRow &R) {
  const int b = A.tiles[tile * ENS_ROWS + (two_d ? 0 : row)];
  int in = b >= 0 ? A.inst[two_d ? 1 : 0][b] : -1;
  if (in >= 0 && A.done[in]) in = -1;
  R.blk = b;
  R.inst = in;
  if (in >= 0) {
    R.solver = A.solver[in];
    R.limiter = A.limiter[in];
    const double qdt = A.dtfactor * A.dt[in];
    for (int d = 0; d < (two_d ? 2 : 1); ++d) {
      const double dx = A.dx[in * 2 + d];
      R.sc[d] = -qdt / dx;
      const double r = A.sa[0].P.cada3_radius * dx;
      R.rd[d] = 1.0 / (r * r);
      R.dxinv[d] = 1.0 / dx;
    }
  }
}

// One face of direction D (run-time, so one copy of the face code serves
// both directions and all call sites) at face coordinates (fi, fj): limited
// reconstruction from the staged primitives, Riemann flux, store to fb.
template <class TF, int ND>
__device__ __forceinline__ uint32_t ens_face_at(const TF *s, const EnsView<TF, ND + 2> &tv, const EnsRow &Rf,
                                                const PhysParams &P, int D, int fi, int fj) {
  constexpr int NW = ND + 2;
  constexpr int FB = (BN16 + 1) * BN16;
  constexpr bool FP64 = sizeof(TF) == 8;
  const TF rd = TF(D == 0 ? Rf.rd[0] : Rf.rd[ND - 1]);
  const int lim = Rf.limiter;
  TF wLp[NW], wRp[NW];
  int base[4], strd[4];
#pragma unroll
  for (int o = 0; o < 4; ++o) tv.addr(D == 0 ? fi + o - 2 : fi, D == 0 ? fj : fj + o - 2, base[o], strd[o]);
#pragma unroll
  for (int v = 0; v < NW; ++v) {
    const int ov = orig_index_rt<false, ND>(v, D);
    TF q[4];
#pragma unroll
    for (int o = 0; o < 4; ++o) q[o] = s[base[o] + ov * strd[o]];
    const TF d0 = q[1] - q[0], d1 = q[2] - q[1], d2 = q[3] - q[2];
    TF ldw, rdw;
    face_slopes<TF, 0, sizeof(TF) == 4>(lim, d0, d1, d2, rd, ldw, rdw);
    wLp[v] = q[1] + TF(0.5) * ldw;
    wRp[v] = q[2] - TF(0.5) * rdw;
  }
  TF Fr[NW];
  uint32_t st;
  if (Rf.solver == SOLVER_HLLC) st = ens_face<TF, ND, SOLVER_HLLC>(wLp, wRp, P, Fr);
  else if (Rf.solver == SOLVER_HLL) st = ens_face<TF, ND, SOLVER_HLL>(wLp, wRp, P, Fr);
  else st = ens_face<TF, ND, SOLVER_TVDLF>(wLp, wRp, P, Fr);
  TF *fb = D == 0 ? tv.fbx : tv.fby;
  const int f = D == 0 ? fj * (BN16 + 1) + fi : fj * BN16 + fi;
  const double sc = D == 0 ? Rf.sc[0] : Rf.sc[ND - 1];
#pragma unroll
  for (int v = 0; v < NW; ++v) {
    const int ov = orig_index_rt<false, ND>(v, D);
    if constexpr (FP64) fb[ov * FB + f] = sc * Fr[v];
    else fb[ov * FB + f] = Fr[v];
  }
  return st;
}

// One RK stage on one tile; `cur` holds this tile's rows, `nxt` receives the
// rows of tile `next` (if < nt).
template <class TF, int ND>
__device__ __forceinline__ uint32_t ens_stage_tile(const EnsArgs &A, TF *s, const EnsRow *cur, EnsRow *nxt,
                                                   int next, int nt, int n2) {
  using V = Vars<false, ND, false>;
  constexpr int NW = V::NW;
  constexpr int FB = (BN16 + 1) * BN16;
  constexpr bool FP64 = sizeof(TF) == 8;
  const StageArgs &S = A.sa[ND - 1];
  const PhysParams &P = S.P;
  const int t = threadIdx.x;
  const bool cell_thread = t < BN16 * BN16;
  const int ci = t & (BN16 - 1), cj = (t >> 4) & (BN16 - 1);
  const int lane = t - BN16 * BN16;  // ninth warp: 0..31
  uint32_t st = 0;
  EnsView<TF, NW> tv(s);
  const EnsRow &R = cur[ND == 2 ? 0 : cj];
  const bool active = cell_thread && R.inst >= 0;
  const int cjj = ND == 2 ? cj : 0;
  // ---- stage: cells, halos, RK combination; the ninth warp fetches the next tile's rows
  if (!cell_thread) {
    if (lane < ENS_ROWS && next < nt) ens_fill_row(A, next, next < n2, lane, nxt[lane]);
  }
  if (active) {
    double w[NW];
    st |= load_prim<false, ND, false, ND>(S, R.blk, ci, cjj, 0, w);
#pragma unroll
    for (int v = 0; v < NW; ++v) tv.ring[v * BN16 * BN16 + cj * BN16 + ci] = TF(w[v]);
  }
  if (t < (ND == 2 ? 128 : 64)) {
    int i, j, row;
    TF *dst;
    int stride;
    if (t < 64) {
      j = t >> 2;
      const int c = t & 3;
      i = c < 2 ? c - 2 : c + BN16 - 2;
      dst = tv.hx + j * 4 + c;
      stride = BN16 * 4;
      row = ND == 2 ? 0 : j;
    } else {
      const int r = (t - 64) >> 4;
      i = (t - 64) & (BN16 - 1);
      j = r < 2 ? r - 2 : r + BN16 - 2;
      dst = tv.hy + r * BN16 + i;
      stride = 4 * BN16;
      row = 0;
    }
    const EnsRow &H = cur[row];
    if (H.inst >= 0) {
      double w[NW];
      st |= load_prim<false, ND, false, ND>(S, H.blk, i, ND == 2 ? j : 0, 0, w);
#pragma unroll
      for (int v = 0; v < NW; ++v) dst[v * stride] = TF(w[v]);
    }
  }
  double acc[NW];
  if (active) {
#pragma unroll
    for (int v = 0; v < NW; ++v) {
      const size_t o = cell_offset<ND>(R.blk, NW, v, ci, cjj, 0);
      const double win = S.uin[o];
      acc[v] = (A.a_base == 0.0) ? win : A.a_base * S.ubase[o] + A.b_in * win;
    }
  }
  __syncthreads();
  // ---- faces of both directions: up to two per thread, one call site
  {
    int nf = 0, fd0 = 0, fi0 = 0, fj0 = 0, fi1 = 0, fj1 = 0;
    const EnsRow *rf = &R;
    if (active) {
      nf = ND;  // x-face (ci, cj) and, in 2-D, y-face (ci, cj)
      fi0 = ci; fj0 = cj; fi1 = ci; fj1 = cj;
    } else if (!cell_thread) {
      if (lane < BN16) {
        rf = &cur[ND == 2 ? 0 : lane];
        nf = rf->inst >= 0 ? 1 : 0;
        fi0 = BN16; fj0 = lane;
      } else if (ND == 2) {
        rf = &cur[0];
        nf = rf->inst >= 0 ? 1 : 0;
        fd0 = 1; fi0 = lane - BN16; fj0 = BN16;
      }
    }
#pragma unroll 1
    for (int q = 0; q < nf; ++q)
      st |= ens_face_at<TF, ND>(s, tv, *rf, P, q == 0 ? fd0 : 1, q == 0 ? fi0 : fi1, q == 0 ? fj0 : fj1);
  }
  __syncthreads();
  // ---- flux divergence in direction order, small values, store
  if (active) {
#pragma unroll
    for (int D = 0; D < ND; ++D) {
      const TF *fb = D == 0 ? tv.fbx : tv.fby;
      const int f = D == 0 ? cj * (BN16 + 1) + ci : cj * BN16 + ci;
      const int step = D == 0 ? 1 : BN16;
      const double sc = FP64 ? 1.0 : R.sc[D];
#pragma unroll
      for (int v = 0; v < NW; ++v) {
        if constexpr (FP64) acc[v] = acc[v] + fb[v * FB + f + step] - fb[v * FB + f];
        else acc[v] = acc[v] + sc * double(fb[v * FB + f + step]) - sc * double(fb[v * FB + f]);
      }
    }
    if (P.fix_small_values) {
      if (small_values<double, false, ND, false>(acc, false, P) && P.small_values_method != 1) st |= ST_SMALL_VALUE;
    }
    if (!isfinite(acc[V::RHO]) || !isfinite(acc[V::E])) {
      st |= ST_NAN;
      atomicOr(A.inst_status + R.inst, ST_NAN);
    }
#pragma unroll
    for (int v = 0; v < NW; ++v) S.uout[cell_offset<ND>(R.blk, NW, v, ci, cjj, 0)] = acc[v];
  }
  return st;
}

template <class TF>
__device__ __forceinline__ void ens_stage_body(const EnsArgs &A) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  TF *sm = reinterpret_cast<TF *>(smem_raw);
  __shared__ EnsRow rows[3][ENS_ROWS];
  const int n2 = A.ntiles[0], nt = A.ntiles[1];
  int tile = blockIdx.x;
  if (tile >= nt) return;
  const int t = threadIdx.x;
  if (t >= BN16 * BN16 && t < BN16 * BN16 + ENS_ROWS) ens_fill_row(A, tile, tile < n2, t - BN16 * BN16, rows[0][t - BN16 * BN16]);
  __syncthreads();
  uint32_t st = 0;
#pragma unroll 1
  for (int k = 0; tile < nt; ++k, tile += gridDim.x) {
    // One shared tile serves every tile: the faces read the cells and halos
    // before the second barrier, the next tile's staging writes them after
    // it; the next tile's faces write the flux buffers only after its first
    // barrier, which every thread reaches after accumulating this tile.  The
    // row table is k % 3 (the ninth warp fills tile k+1's while tile k runs).
    TF *s = sm;
    const EnsRow *cur = rows[k % 3];
    EnsRow *nxt = rows[(k + 1) % 3];
    const int next = tile + gridDim.x;
    if (tile < n2) st |= ens_stage_tile<TF, 2>(A, s, cur, nxt, next, nt, n2);
    else st |= ens_stage_tile<TF, 1>(A, s, cur, nxt, next, nt, n2);
  }
  if (st) atomicOr(A.sa[0].status, st);
}

// Occupancy: two CTAs of 288 threads per SM in FP64 (96 registers: 18 warps
// put five on one SM sub-partition, whose 16 K registers then cap a thread at
// 102), three in the mixed form (72 registers, measured 1.23x faster than two).
// Denser variants, which the autotuner times against the first kernel of a
// form: FP64 at three CTAs per SM (72 registers, a few spilled) and four (56),
// mixed at four (56 registers) and five (40).
__global__ void __launch_bounds__(ENS_THREADS, 2) ens_stage_kernel_fp64(const EnsArgs A) { ens_stage_body<double>(A); }
__global__ void __launch_bounds__(ENS_THREADS, 3) ens_stage_kernel_fp64_3(const EnsArgs A) { ens_stage_body<double>(A); }
__global__ void __launch_bounds__(ENS_THREADS, 4) ens_stage_kernel_fp64_4(const EnsArgs A) { ens_stage_body<double>(A); }
__global__ void __launch_bounds__(ENS_THREADS, 3) ens_stage_kernel_mixed(const EnsArgs A) { ens_stage_body<float>(A); }
__global__ void __launch_bounds__(ENS_THREADS, 4) ens_stage_kernel_mixed_4(const EnsArgs A) { ens_stage_body<float>(A); }
__global__ void __launch_bounds__(ENS_THREADS, 5) ens_stage_kernel_mixed_5(const EnsArgs A) { ens_stage_body<float>(A); }

// the stage kernel of (precision, variant); variant v is capped for
// ens_variant_ctas(mixed, v) CTAs per SM
static void (*ens_stage_fn(bool mixed, int var))(const EnsArgs) {
  if (mixed) return var == 2 ? ens_stage_kernel_mixed_5 : (var == 1 ? ens_stage_kernel_mixed_4 : ens_stage_kernel_mixed);
  return var == 2 ? ens_stage_kernel_fp64_4 : (var == 1 ? ens_stage_kernel_fp64_3 : ens_stage_kernel_fp64);
}
static int ens_variants(bool) { return 3; }
static int ens_variant_ctas(bool mixed, int var) { return (mixed ? 3 : 2) + var; }

// getdt_courant (src/mod_dt.t:160-287), maxsum, per instance: the max over
// the instance's cells of sum_d (|v_d| + c_s) / dx_d.
template <int ND>
__device__ __forceinline__ void ens_getdt_tile(const EnsArgs &A, int tile, EnsRow *rows, double *wred) {
  using V = Vars<false, ND, false>;
  constexpr int NW = V::NW;
  const StageArgs &S = A.sa[ND - 1];
  const int t = threadIdx.x;
  const int ci = t & (BN16 - 1), cj = t >> 4;
  if (!ens_rows<ND>(A, tile, true, rows)) {
    __syncthreads();
    return;
  }
  const EnsRow &R = rows[ND == 2 ? 0 : cj];
  double x = 0.0;
  if (R.inst >= 0) {
    double w[NW];
#pragma unroll
    for (int v = 0; v < NW; ++v) w[v] = __ldg(S.uin + cell_offset<ND>(R.blk, NW, v, ci, ND == 2 ? cj : 0, 0));
    // phys_to_primitive with its small-value fix (src/mod_dt.t:189-191)
    if (S.P.fix_small_values) {
      if (small_values<double, false, ND, false>(w, false, S.P) && S.P.small_values_method != 1)
        atomicOr(A.inst_status + R.inst, ST_SMALL_VALUE);
    }
    to_primitive<false, ND, false>(w, S.P);
#pragma unroll
    for (int d = 0; d < ND; ++d) {
      const double cm = fabs(w[V::M0 + d]) + sqrt(S.P.gamma * w[V::E] / w[V::RHO]);
      const double c = cm * R.dxinv[d];
      x = d == 0 ? c : x + c;
    }
  }
  // rows are half-warps: reduce over the 16 lanes of a row
#pragma unroll
  for (int o = 8; o > 0; o >>= 1) x = fmax(x, __shfl_xor_sync(0xffffffffu, x, o));
  if constexpr (ND == 1) {
    if (ci == 0 && R.inst >= 0) atomic_max_pos(A.red + R.inst, x);
  } else {
    if (ci == 0) wred[cj] = x;
    __syncthreads();
    if (t == 0 && R.inst >= 0) {
      double m = 0.0;
      for (int q = 0; q < ENS_ROWS; ++q) m = fmax(m, wred[q]);
      atomic_max_pos(A.red + R.inst, m);
    }
  }
  __syncthreads();
}

__global__ void __launch_bounds__(STAGE_THREADS) ens_getdt_kernel(const EnsArgs A) {
  __shared__ EnsRow rows[ENS_ROWS];
  __shared__ double wred[ENS_ROWS];
  const int n2 = A.ntiles[0], nt = A.ntiles[1];
#pragma unroll 1
  for (int tile = blockIdx.x; tile < nt; tile += gridDim.x) {
    if (tile < n2) ens_getdt_tile<2>(A, tile, rows, wred);
    else ens_getdt_tile<1>(A, tile, rows, wred);
  }
}

struct EnsTime {
  int ninst;
  unsigned long long *red;
  double *dt, *time;
  const double *time_max;
  int *done, *steps;
  uint32_t *inst_status, *status;
  double courantpar, dtmin;
};

// setdt per instance (src/mod_dt.t:30-79) and the exit test of the time loop
// (src/amrvac.t:306: global_time >= time_max or final_dt_exit).
__global__ void ens_finalize_kernel(const EnsTime T) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= T.ninst) return;
  const double x = __longlong_as_double((long long)T.red[i]);
  T.red[i] = 0ull;
  if (T.done[i]) { T.dt[i] = 0.0; return; }
  // An instance whose last step produced a non-finite density or energy (or
  // a small-value error) stops here with that status; the others go on.
  if (T.inst_status[i] & (ST_SMALL_VALUE | ST_NAN)) {
    atomicOr(T.status, T.inst_status[i]);
    T.done[i] = 1;
    T.dt[i] = 0.0;
    return;
  }
  double d = 1.0e99;
  if (x > 1.0e-12) d = fmin(d, T.courantpar / x);
  const double t = T.time[i], tmax = T.time_max[i];
  if (d < T.dtmin) {  // crash: this instance stops
    T.inst_status[i] |= ST_DT_TOO_SMALL;
    atomicOr(T.status, ST_DT_TOO_SMALL);
    T.done[i] = 1;
    T.dt[i] = 0.0;
    return;
  }
  if (tmax - t <= T.dtmin || t >= tmax) {
    T.done[i] = 1;
    T.dt[i] = 0.0;
    return;
  }
  T.dt[i] = fmin(d, tmax - t);
}

__global__ void ens_advance_kernel(const EnsTime T) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= T.ninst || T.done[i]) return;
  T.time[i] = T.time[i] + T.dt[i];
  T.steps[i] += 1;
}

}  // namespace amrvac

using namespace amrvac;

struct amrvac_ens {
  amrvac_cfg cfg;
  PhysParams P;
  BcSpec bc;
  SrlMaps maps;
  bool mixed = false;
  int ninst = 0;
  std::vector<amrvac_ens_instance> inst;
  std::vector<int> pool_of, first, nblk;     // per instance: pool (0: 1-D, 1: 2-D), first block, blocks
  std::vector<int> h_tiles2, h_tiles1;       // 2-D tiles (one block each), 1-D tiles (16 rows)
  std::vector<std::vector<int>> tiles1_of;   // 1-D tile indices per instance (for compaction)
  int nb[2] = {0, 0};
  double *pool[2][3] = {{nullptr, nullptr, nullptr}, {nullptr, nullptr, nullptr}};
  int *d_nbr[2] = {nullptr, nullptr};
  int *d_inst[2] = {nullptr, nullptr};
  int *d_tiles = nullptr, *d_ntiles = nullptr;
  int ntiles_active[2] = {0, 0};
  double *d_dt = nullptr, *d_time = nullptr, *d_tmax = nullptr, *d_dx = nullptr;
  int *d_solver = nullptr, *d_limiter = nullptr, *d_done = nullptr, *d_steps = nullptr;
  unsigned long long *d_red = nullptr;
  uint32_t *d_status = nullptr, *d_inst_status = nullptr;
  double *d_stage = nullptr;
  size_t stage_doubles = 0;
  int *h_pin = nullptr;                      // pinned: ntiles + tile list for compaction uploads
  size_t h_pin_ints = 0;
  std::vector<int> h_done;
  cudaStream_t stream = nullptr;
  cudaGraphExec_t graph = nullptr;
  int graph_steps = 0;
  int grid = 0;          // CTAs per stage / getdt launch
  int wave = 1;          // resident stage CTAs of the current variant
  int var = 0;           // stage-kernel variant: each one CTA per SM denser than the last
  int nvar = 2;
  int wave_v[3] = {1, 1, 1};
  int64_t launches = 0;
};

namespace {

int efail(int code, const std::string &m) { return record_error(code, "ens: " + m); }
int ecuda(cudaError_t e, const char *where) {
  return record_error(AMRVAC_E_CUDA, std::string("ens: ") + where + ": " + cudaGetErrorString(e));
}
#define ECK(call)                                   \
  do {                                              \
    cudaError_t e_ = (call);                        \
    if (e_ != cudaSuccess) return ecuda(e_, #call); \
  } while (0)

size_t ens_smem(bool mixed) {
  return mixed ? sizeof(float) * EnsTile<float>::TOTAL : sizeof(double) * EnsTile<double>::TOTAL;
}

EnsArgs ens_args(amrvac_ens *e, int reg_ct, int reg_new, int reg_base, double a, double b, double dtfactor) {
  EnsArgs A;
  std::memset(&A, 0, sizeof(A));
  for (int p = 0; p < 2; ++p) {
    StageArgs &S = A.sa[p];
    S.uin = e->pool[p][reg_ct];
    S.ubase = e->pool[p][reg_base];
    S.uout = e->pool[p][reg_new];
    S.nbr = e->d_nbr[p];
    S.nblocks = e->nb[p];
    for (int s = 0; s < 6; ++s) { S.bc_kind[s] = e->bc.kind[s]; S.bc_flip[s] = 0; }
    S.status = e->d_status;
    S.P = e->P;
    A.inst[p] = e->d_inst[p];
  }
  A.tiles = e->d_tiles;
  A.ntiles = e->d_ntiles;
  A.a_base = a;
  A.b_in = b;
  A.dtfactor = dtfactor;
  A.dt = e->d_dt;
  A.dx = e->d_dx;
  A.solver = e->d_solver;
  A.limiter = e->d_limiter;
  A.done = e->d_done;
  A.red = e->d_red;
  A.inst_status = e->d_inst_status;
  return A;
}

EnsTime ens_time(amrvac_ens *e) {
  EnsTime T;
  T.ninst = e->ninst;
  T.red = e->d_red;
  T.dt = e->d_dt;
  T.time = e->d_time;
  T.time_max = e->d_tmax;
  T.done = e->d_done;
  T.steps = e->d_steps;
  T.inst_status = e->d_inst_status;
  T.status = e->d_status;
  T.courantpar = e->cfg.courantpar;
  T.dtmin = e->cfg.dtmin;
  return T;
}

int ens_launch_stage(amrvac_ens *e, int reg_ct, int reg_new, int reg_base, double a, double b, double dtf) {
  const EnsArgs A = ens_args(e, reg_ct, reg_new, reg_base, a, b, dtf);
  ens_stage_fn(e->mixed, e->var)<<<e->grid, ENS_THREADS, ens_smem(e->mixed), e->stream>>>(A);
  ECK(cudaGetLastError());
  ++e->launches;
  return 0;
}

int ens_launch_step(amrvac_ens *e) {
  const EnsArgs G = ens_args(e, 0, 0, 0, 0.0, 1.0, 1.0);
  ens_getdt_kernel<<<e->grid, STAGE_THREADS, 0, e->stream>>>(G);
  ECK(cudaGetLastError());
  const EnsTime T = ens_time(e);
  const int nb = (e->ninst + 127) / 128;
  ens_finalize_kernel<<<nb, 128, 0, e->stream>>>(T);
  ECK(cudaGetLastError());
  e->launches += 2;
  const amrvac_cfg &k = e->cfg;
  int r = 0;
  if (k.time_stepper == AMRVAC_TS_ONESTEP) {
    for (int p = 0; p < 2; ++p)
      if (e->nb[p])
        ECK(cudaMemcpyAsync(e->pool[p][1], e->pool[p][0], sizeof(double) * (size_t)e->nb[p] * (p ? 4 * 256 : 3 * 16),
                            cudaMemcpyDeviceToDevice, e->stream));
    r = ens_launch_stage(e, 1, 0, 0, 0.0, 1.0, 1.0);
  } else if (k.time_stepper == AMRVAC_TS_TWOSTEP) {
    if ((r = ens_launch_stage(e, 0, 1, 0, 0.0, 1.0, 1.0))) return r;
    r = ens_launch_stage(e, 1, 0, 0, 0.5, 0.5, 0.5);
  } else {
    double b11, b22, b33, a21, a31;
    if (k.ssprk_order == 2) { b11 = 0.5; b22 = 0.5; b33 = 1.0 / 3.0; a21 = 0.0; a31 = 1.0 / 3.0; }
    else { b11 = 1.0; b22 = 1.0 / 4.0; b33 = 2.0 / 3.0; a21 = 3.0 / 4.0; a31 = 1.0 / 3.0; }
    if ((r = ens_launch_stage(e, 0, 1, 0, 0.0, 1.0, b11))) return r;
    if ((r = ens_launch_stage(e, 1, 2, 0, a21, 1.0 - a21, b22))) return r;
    r = ens_launch_stage(e, 2, 0, 0, a31, 1.0 - a31, b33);
  }
  if (r) return r;
  ens_advance_kernel<<<nb, 128, 0, e->stream>>>(T);
  ECK(cudaGetLastError());
  ++e->launches;
  return 0;
}

// Upload the tile list of the instances not yet done (done == nullptr: all).
int ens_upload_tiles(amrvac_ens *e, const std::vector<int> *done) {
  std::vector<int> t2, t1;
  t2.reserve(e->h_tiles2.size());
  for (int i = 0; i < e->ninst; ++i) {
    if (done && (*done)[i]) continue;
    if (e->pool_of[i] == 1)
      for (int b = 0; b < e->nblk[i]; ++b) t2.push_back(e->first[i] + b);
  }
  std::vector<char> keep(e->h_tiles1.size() / ENS_ROWS, 0);
  for (int i = 0; i < e->ninst; ++i)
    if (e->pool_of[i] == 0 && !(done && (*done)[i]))
      for (int q : e->tiles1_of[i]) keep[q] = 1;
  const size_t n2 = t2.size();
  size_t n1 = 0;
  for (char c : keep) n1 += c;
  const size_t total = n2 + n1;
  if (total + 1 > e->h_pin_ints / ENS_ROWS) return efail(AMRVAC_E_STATE, "tile staging too small");
  // pinned staging: [0..15] ntiles, then the tiles; the previous upload from it has completed
  // (the caller synchronised the stream)
  int *h = e->h_pin;
  h[0] = (int)n2;
  h[1] = (int)total;
  int *dst = h + ENS_ROWS;
  for (size_t q = 0; q < n2; ++q) {
    dst[q * ENS_ROWS] = t2[q];
    for (int r = 1; r < ENS_ROWS; ++r) dst[q * ENS_ROWS + r] = -1;
  }
  size_t w = n2;
  for (size_t q = 0; q < keep.size(); ++q) {
    if (!keep[q]) continue;
    std::memcpy(dst + w * ENS_ROWS, e->h_tiles1.data() + q * ENS_ROWS, sizeof(int) * ENS_ROWS);
    ++w;
  }
  ECK(cudaMemcpyAsync(e->d_ntiles, h, sizeof(int) * 2, cudaMemcpyHostToDevice, e->stream));
  if (total)
    ECK(cudaMemcpyAsync(e->d_tiles, dst, sizeof(int) * total * ENS_ROWS, cudaMemcpyHostToDevice, e->stream));
  ECK(cudaStreamSynchronize(e->stream));
  e->ntiles_active[0] = (int)n2;
  e->ntiles_active[1] = (int)total;
  return 0;
}

int ens_ensure_stage(amrvac_ens *e, size_t doubles) {
  if (e->stage_doubles >= doubles) return 0;
  cudaStreamSynchronize(e->stream);
  cudaFree(e->d_stage);
  e->d_stage = nullptr;
  e->stage_doubles = 0;
  ECK(cudaMalloc(&e->d_stage, sizeof(double) * doubles));
  e->stage_doubles = doubles;
  return 0;
}

void free_all(amrvac_ens *e) {
  if (e->graph) cudaGraphExecDestroy(e->graph);
  for (int p = 0; p < 2; ++p) {
    for (int r = 0; r < 3; ++r) cudaFree(e->pool[p][r]);
    cudaFree(e->d_nbr[p]);
    cudaFree(e->d_inst[p]);
  }
  cudaFree(e->d_tiles); cudaFree(e->d_ntiles);
  cudaFree(e->d_dt); cudaFree(e->d_time); cudaFree(e->d_tmax); cudaFree(e->d_dx);
  cudaFree(e->d_solver); cudaFree(e->d_limiter); cudaFree(e->d_done); cudaFree(e->d_steps);
  cudaFree(e->d_red); cudaFree(e->d_status); cudaFree(e->d_inst_status); cudaFree(e->d_stage);
  if (e->h_pin) cudaFreeHost(e->h_pin);
  if (e->stream) cudaStreamDestroy(e->stream);
}

int check_ens(amrvac_ens *e) { return e ? 0 : efail(AMRVAC_E_ARG, "null ensemble"); }

int check_inst(amrvac_ens *e, int i) {
  if (int r = check_ens(e)) return r;
  if (i < 0 || i >= e->ninst) return efail(AMRVAC_E_ARG, "instance out of range");
  return 0;
}

}  // namespace

extern "C" {

int amrvac_ens_create(const amrvac_cfg *cfg, int ninst, const amrvac_ens_instance *in, amrvac_ens **out) {
  if (!cfg || !in || !out) return efail(AMRVAC_E_ARG, "null argument");
  *out = nullptr;
  if (ninst <= 0) return efail(AMRVAC_E_ARG, "ninst must be positive");
  const amrvac_cfg &k = *cfg;
  if (k.physics != 0) return efail(AMRVAC_E_UNSUPPORTED, "ensembles are hydrodynamics (physics 0) only");
  if (k.nghostcells < 2) return efail(AMRVAC_E_UNSUPPORTED, "nghostcells must be >= 2");
  if (k.type_courant != AMRVAC_COURANT_MAXSUM) return efail(AMRVAC_E_UNSUPPORTED, "ensembles use typecourant maxsum");
  if (k.typeboundspeed < 1 || k.typeboundspeed > 3) return efail(AMRVAC_E_ARG, "bad typeboundspeed");
  if (k.time_stepper < 1 || k.time_stepper > 3) return efail(AMRVAC_E_UNSUPPORTED, "time_stepper not supported");
  if (k.time_stepper == AMRVAC_TS_TWOSTEP && k.time_integrator != AMRVAC_TI_SSPRK2)
    return efail(AMRVAC_E_UNSUPPORTED, "ensembles: twostep with time_integrator ssprk2 only");
  if (k.precision != 0 && k.precision != 1) return efail(AMRVAC_E_ARG, "precision must be 0 or 1");
  if (k.fix_small_values && k.small_values_method == 2)
    return efail(AMRVAC_E_UNSUPPORTED, "ensembles: small_values_method error or replace");
  for (int s = 0; s < 4; ++s)
    for (int v = 0; v < 4; ++v) {
      const int b = k.typeboundary[s][v];
      if (b != k.typeboundary[s][0] || (b != AMRVAC_BC_PERIODIC && b != AMRVAC_BC_CONT))
        return efail(AMRVAC_E_UNSUPPORTED, "ensemble boundaries: periodic or cont, the same for all variables");
    }
  for (int i = 0; i < ninst; ++i) {
    const amrvac_ens_instance &q = in[i];
    if (q.ndim != 1 && q.ndim != 2) return efail(AMRVAC_E_UNSUPPORTED, "instance ndim must be 1 or 2");
    for (int d = 0; d < q.ndim; ++d) {
      if (q.domain_nx[d] <= 0 || q.domain_nx[d] % 16) return efail(AMRVAC_E_ARG, "domain_nx must be a positive multiple of 16");
      if (!(q.xprobmax[d] > q.xprobmin[d])) return efail(AMRVAC_E_ARG, "xprobmax must exceed xprobmin");
    }
    if (q.flux_scheme != AMRVAC_FS_TVDLF && q.flux_scheme != AMRVAC_FS_HLL && q.flux_scheme != AMRVAC_FS_HLLC)
      return efail(AMRVAC_E_UNSUPPORTED, "instance flux_scheme must be tvdlf, hll or hllc");
    if (q.limiter < 1 || q.limiter > 9) return efail(AMRVAC_E_UNSUPPORTED, "limiter not supported");
  }
  amrvac_ens *e = new amrvac_ens();
  e->cfg = k;
  e->mixed = k.precision == 1;
  e->ninst = ninst;
  e->inst.assign(in, in + ninst);
  PhysParams &P = e->P;
  std::memset(&P, 0, sizeof(P));
  P.gamma = k.gamma;
  P.gamma_1 = k.gamma - 1.0;
  P.inv_gamma_1 = 1.0 / (k.gamma - 1.0);
  P.small_density = k.small_density;
  P.small_pressure = k.small_pressure;
  P.small_e = k.small_pressure / (k.gamma - 1.0);
  P.tvdlfeps = k.tvdlfeps;
  P.cada3_radius = k.cada3_radius;
  for (int d = 0; d < 3; ++d) P.schmid_rad[d] = 1.0;  // the ensemble takes no schmid limiter
  P.schmid_global = 0;
  P.courantpar = k.courantpar;
  P.limiter = 0;
  P.boundspeed = k.typeboundspeed;
  P.fix_small_values = k.fix_small_values;
  P.check_small_values = k.check_small_values;
  P.small_values_method = k.small_values_method;
  for (int s = 0; s < 6; ++s) {
    e->bc.kind[s] = s < 4 && k.typeboundary[s][0] == AMRVAC_BC_CONT ? BCK_CONT : BCK_PERIODIC;
    e->bc.flip[s] = 0;
  }
  for (int d = 0; d < 3; ++d) {
    if (d < 2) amrvac_gpu_srl_maps(k.nghostcells, 16, e->maps.smin[d], e->maps.smax[d], e->maps.rmin[d], e->maps.rmax[d]);
    else for (int q = 0; q < 3; ++q) e->maps.smin[d][q] = e->maps.smax[d][q] = e->maps.rmin[d][q] = e->maps.rmax[d][q] = 0;
  }
  // ---- blocks and neighbour tables
  std::vector<int> nbr[2], binst[2];
  std::vector<double> dxv(2 * (size_t)ninst, 1.0);
  e->pool_of.resize(ninst);
  e->first.resize(ninst);
  e->nblk.resize(ninst);
  for (int i = 0; i < ninst; ++i) {
    const amrvac_ens_instance &q = in[i];
    const int p = q.ndim - 1;
    const int nbx = q.domain_nx[0] / 16, nby = q.ndim == 2 ? q.domain_nx[1] / 16 : 1;
    e->pool_of[i] = p;
    e->first[i] = e->nb[p];
    e->nblk[i] = nbx * nby;
    for (int d = 0; d < q.ndim; ++d) dxv[2 * i + d] = (q.xprobmax[d] - q.xprobmin[d]) / q.domain_nx[d];
    for (int jb = 0; jb < nby; ++jb)
      for (int ib = 0; ib < nbx; ++ib) {
        for (int dk = -1; dk <= 1; ++dk)
          for (int dj = -1; dj <= 1; ++dj)
            for (int di = -1; di <= 1; ++di) {
              int v = -1;
              if (dk == 0 && (q.ndim == 2 || dj == 0)) {
                int x = ib + di, y = jb + dj;
                bool ok = true;
                if (x < 0 || x >= nbx) {
                  if (e->bc.kind[x < 0 ? 0 : 1] == BCK_PERIODIC) x = (x + nbx) % nbx;
                  else ok = false;
                }
                if (y < 0 || y >= nby) {
                  if (q.ndim == 2 && e->bc.kind[y < 0 ? 2 : 3] == BCK_PERIODIC) y = (y + nby) % nby;
                  else ok = false;
                }
                if (ok) v = e->first[i] + x + nbx * y;
              }
              nbr[p].push_back(v);
            }
        binst[p].push_back(i);
      }
    e->nb[p] += e->nblk[i];
  }
  // ---- tiles: 2-D blocks one per tile; 1-D blocks packed 16 per tile, grouped by scheme
  for (int i = 0; i < ninst; ++i)
    if (e->pool_of[i] == 1)
      for (int b = 0; b < e->nblk[i]; ++b) e->h_tiles2.push_back(e->first[i] + b);
  std::vector<int> order;
  for (int i = 0; i < ninst; ++i)
    if (e->pool_of[i] == 0) order.push_back(i);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
    const int ka = in[a].flux_scheme * 16 + in[a].limiter, kb = in[b].flux_scheme * 16 + in[b].limiter;
    return ka < kb;
  });
  e->tiles1_of.assign(ninst, {});
  int row = 0;
  for (int i : order)
    for (int b = 0; b < e->nblk[i]; ++b) {
      if (row == 0) e->h_tiles1.insert(e->h_tiles1.end(), ENS_ROWS, -1);
      const int tq = (int)(e->h_tiles1.size() / ENS_ROWS) - 1;
      e->h_tiles1[(size_t)tq * ENS_ROWS + row] = e->first[i] + b;
      if (e->tiles1_of[i].empty() || e->tiles1_of[i].back() != tq) e->tiles1_of[i].push_back(tq);
      row = (row + 1) % ENS_ROWS;
    }
  const size_t ntiles = e->h_tiles2.size() + e->h_tiles1.size() / ENS_ROWS;
  // ---- device memory
  cudaError_t ce;
#define EALLOC(ptr, bytes)                                           \
  if ((ce = cudaMalloc(&(ptr), (bytes))) != cudaSuccess) {           \
    free_all(e);                                                     \
    delete e;                                                        \
    return ecuda(ce, "cudaMalloc");                                  \
  }
  if ((ce = cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking)) != cudaSuccess) {
    delete e;
    return ecuda(ce, "cudaStreamCreate");
  }
  for (int p = 0; p < 2; ++p) {
    if (!e->nb[p]) continue;
    const size_t per = p ? 4 * 256 : 3 * 16;
    for (int r = 0; r < 3; ++r) EALLOC(e->pool[p][r], sizeof(double) * per * e->nb[p]);
    EALLOC(e->d_nbr[p], sizeof(int) * nbr[p].size());
    EALLOC(e->d_inst[p], sizeof(int) * binst[p].size());
  }
  EALLOC(e->d_tiles, sizeof(int) * ENS_ROWS * std::max<size_t>(ntiles, 1));
  EALLOC(e->d_ntiles, sizeof(int) * 2);
  EALLOC(e->d_dt, sizeof(double) * ninst);
  EALLOC(e->d_time, sizeof(double) * ninst);
  EALLOC(e->d_tmax, sizeof(double) * ninst);
  EALLOC(e->d_dx, sizeof(double) * 2 * ninst);
  EALLOC(e->d_solver, sizeof(int) * ninst);
  EALLOC(e->d_limiter, sizeof(int) * ninst);
  EALLOC(e->d_done, sizeof(int) * ninst);
  EALLOC(e->d_steps, sizeof(int) * ninst);
  EALLOC(e->d_red, sizeof(unsigned long long) * ninst);
  EALLOC(e->d_status, sizeof(uint32_t));
  EALLOC(e->d_inst_status, sizeof(uint32_t) * ninst);
#undef EALLOC
  e->h_pin_ints = (ntiles + 1) * ENS_ROWS;
  if ((ce = cudaMallocHost(&e->h_pin, sizeof(int) * e->h_pin_ints)) != cudaSuccess) {
    free_all(e);
    delete e;
    return ecuda(ce, "cudaMallocHost");
  }
  std::vector<double> tmax(ninst);
  std::vector<int> solver(ninst), lim(ninst);
  for (int i = 0; i < ninst; ++i) {
    tmax[i] = in[i].time_max;
    solver[i] = in[i].flux_scheme;  // AMRVAC_FS_* equal SOLVER_*
    lim[i] = in[i].limiter;
  }
  auto fail_free = [&](cudaError_t c2, const char *w) {
    free_all(e);
    delete e;
    return ecuda(c2, w);
  };
  for (int p = 0; p < 2; ++p) {
    if (!e->nb[p]) continue;
    if ((ce = cudaMemcpy(e->d_nbr[p], nbr[p].data(), sizeof(int) * nbr[p].size(), cudaMemcpyHostToDevice)) ||
        (ce = cudaMemcpy(e->d_inst[p], binst[p].data(), sizeof(int) * binst[p].size(), cudaMemcpyHostToDevice)))
      return fail_free(ce, "cudaMemcpy(tables)");
  }
  if ((ce = cudaMemcpy(e->d_tmax, tmax.data(), sizeof(double) * ninst, cudaMemcpyHostToDevice)) ||
      (ce = cudaMemcpy(e->d_dx, dxv.data(), sizeof(double) * 2 * ninst, cudaMemcpyHostToDevice)) ||
      (ce = cudaMemcpy(e->d_solver, solver.data(), sizeof(int) * ninst, cudaMemcpyHostToDevice)) ||
      (ce = cudaMemcpy(e->d_limiter, lim.data(), sizeof(int) * ninst, cudaMemcpyHostToDevice)) ||
      (ce = cudaMemset(e->d_red, 0, sizeof(unsigned long long) * ninst)) ||
      (ce = cudaMemset(e->d_status, 0, sizeof(uint32_t))))
    return fail_free(ce, "cudaMemcpy(instances)");
  for (int p = 0; p < 2; ++p)
    for (int r = 0; r < 3; ++r)
      if (e->pool[p][r] && (ce = cudaMemset(e->pool[p][r], 0, sizeof(double) * (p ? 4 * 256 : 3 * 16) * e->nb[p])))
        return fail_free(ce, "cudaMemset(pool)");
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  e->nvar = ens_variants(e->mixed);
  for (int v = 0; v < e->nvar; ++v) {
    ce = cudaFuncSetAttribute(ens_stage_fn(e->mixed, v), cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)ens_smem(e->mixed));
    if (ce) return fail_free(ce, "cudaFuncSetAttribute");
    int per_sm = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ens_stage_fn(e->mixed, v), ENS_THREADS,
                                                  ens_smem(e->mixed));
    e->wave_v[v] = std::max(1, per_sm) * nsm;
  }
  e->var = 0;
  e->wave = e->wave_v[0];
  e->grid = e->wave;
  *out = e;
  if (int r = amrvac_ens_reset_time(e)) {
    *out = nullptr;
    free_all(e);
    delete e;
    return r;
  }
  return 0;
}

int amrvac_ens_destroy(amrvac_ens *e) {
  if (!e) return 0;
  cudaStreamSynchronize(e->stream);
  free_all(e);
  delete e;
  return 0;
}

int amrvac_ens_nblocks(const amrvac_ens *e, int inst) {
  if (!e || inst < 0 || inst >= e->ninst) return AMRVAC_E_ARG;
  return e->nblk[inst];
}

int amrvac_ens_reset_time(amrvac_ens *e) {
  if (int r = check_ens(e)) return r;
  ECK(cudaMemsetAsync(e->d_time, 0, sizeof(double) * e->ninst, e->stream));
  ECK(cudaMemsetAsync(e->d_dt, 0, sizeof(double) * e->ninst, e->stream));
  ECK(cudaMemsetAsync(e->d_done, 0, sizeof(int) * e->ninst, e->stream));
  ECK(cudaMemsetAsync(e->d_steps, 0, sizeof(int) * e->ninst, e->stream));
  ECK(cudaMemsetAsync(e->d_inst_status, 0, sizeof(uint32_t) * e->ninst, e->stream));
  ECK(cudaMemsetAsync(e->d_red, 0, sizeof(unsigned long long) * e->ninst, e->stream));
  ECK(cudaStreamSynchronize(e->stream));
  return ens_upload_tiles(e, nullptr);
}

int amrvac_ens_upload(amrvac_ens *e, int inst, const double *w) {
  if (int r = check_inst(e, inst)) return r;
  if (!w) return efail(AMRVAC_E_ARG, "null array");
  const int p = e->pool_of[inst], nw = p ? 4 : 3, ndim = p + 1;
  const size_t g = (size_t)(16 + 2 * e->cfg.nghostcells) * (p ? 16 + 2 * e->cfg.nghostcells : 1);
  const size_t doubles = g * nw * e->nblk[inst];
  if (int r = ens_ensure_stage(e, doubles)) return r;
  ECK(cudaMemcpyAsync(e->d_stage, w, sizeof(double) * doubles, cudaMemcpyHostToDevice, e->stream));
  ECK(launch_unpack(e->d_stage, e->pool[p][0], e->first[inst], e->nblk[inst], nw, ndim, e->cfg.nghostcells, BN16,
                    e->stream));
  ++e->launches;
  ECK(cudaStreamSynchronize(e->stream));
  return 0;
}

int amrvac_ens_download(amrvac_ens *e, int inst, double *w) {
  if (int r = check_inst(e, inst)) return r;
  if (!w) return efail(AMRVAC_E_ARG, "null array");
  const int p = e->pool_of[inst], nw = p ? 4 : 3, ndim = p + 1;
  const size_t g = (size_t)(16 + 2 * e->cfg.nghostcells) * (p ? 16 + 2 * e->cfg.nghostcells : 1);
  const size_t doubles = g * nw * e->nblk[inst];
  if (int r = ens_ensure_stage(e, doubles)) return r;
  ECK(launch_pack(e->pool[p][0], e->d_stage, e->first[inst], e->nblk[inst], nw, ndim, e->cfg.nghostcells, BN16,
                  e->d_nbr[p], e->maps, e->bc, nullptr, e->stream));
  ++e->launches;
  ECK(cudaMemcpyAsync(w, e->d_stage, sizeof(double) * doubles, cudaMemcpyDeviceToHost, e->stream));
  ECK(cudaStreamSynchronize(e->stream));
  return 0;
}

int amrvac_ens_step(amrvac_ens *e) {
  if (int r = check_ens(e)) return r;
  return ens_launch_step(e);
}

int amrvac_ens_run(amrvac_ens *e, int max_steps, int chunk, int *steps_taken, int *nactive) {
  if (int r = check_ens(e)) return r;
  if (max_steps <= 0) return efail(AMRVAC_E_ARG, "max_steps must be positive");
  if (chunk <= 0) chunk = 16;
  if (e->graph && e->graph_steps != chunk) {
    cudaGraphExecDestroy(e->graph);
    e->graph = nullptr;
  }
  if (!e->graph) {
    cudaGraph_t g;
    const int64_t before = e->launches;
    ECK(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
    int r = 0;
    for (int s = 0; s < chunk && !r; ++s) r = ens_launch_step(e);
    cudaError_t ce = cudaStreamEndCapture(e->stream, &g);
    e->launches = before;
    if (r) { if (ce == cudaSuccess) cudaGraphDestroy(g); return r; }
    if (ce != cudaSuccess) return ecuda(ce, "cudaStreamEndCapture");
    ce = cudaGraphInstantiate(&e->graph, g, 0);
    cudaGraphDestroy(g);
    if (ce != cudaSuccess) { e->graph = nullptr; return ecuda(ce, "cudaGraphInstantiate"); }
    e->graph_steps = chunk;
  }
  const int per_step = 3 + e->cfg.time_stepper;
  int taken = 0, act = e->ninst;
  e->h_done.assign(e->ninst, 0);
  int ndone_prev = 0;
  while (taken < max_steps) {
    ECK(cudaGraphLaunch(e->graph, e->stream));
    e->launches += (int64_t)chunk * per_step;
    taken += chunk;
    ECK(cudaMemcpyAsync(e->h_done.data(), e->d_done, sizeof(int) * e->ninst, cudaMemcpyDeviceToHost, e->stream));
    ECK(cudaStreamSynchronize(e->stream));
    const int ndone = (int)std::count_if(e->h_done.begin(), e->h_done.end(), [](int d) { return d != 0; });
    act = e->ninst - ndone;
    if (act == 0) break;
    if (ndone != ndone_prev) {  // drop the finished instances' tiles
      if (int r = ens_upload_tiles(e, &e->h_done)) return r;
      ndone_prev = ndone;
    }
  }
  if (steps_taken) *steps_taken = taken;
  if (nactive) *nactive = act;
  return 0;
}

int amrvac_ens_state(amrvac_ens *e, double *t, double *dt, int *steps, int *done) {
  if (int r = check_ens(e)) return r;
  if (t) ECK(cudaMemcpyAsync(t, e->d_time, sizeof(double) * e->ninst, cudaMemcpyDeviceToHost, e->stream));
  if (dt) ECK(cudaMemcpyAsync(dt, e->d_dt, sizeof(double) * e->ninst, cudaMemcpyDeviceToHost, e->stream));
  if (steps) ECK(cudaMemcpyAsync(steps, e->d_steps, sizeof(int) * e->ninst, cudaMemcpyDeviceToHost, e->stream));
  if (done) ECK(cudaMemcpyAsync(done, e->d_done, sizeof(int) * e->ninst, cudaMemcpyDeviceToHost, e->stream));
  ECK(cudaStreamSynchronize(e->stream));
  return 0;
}

int amrvac_ens_status(amrvac_ens *e, uint32_t *flags, uint32_t *inst_flags) {
  if (int r = check_ens(e)) return r;
  if (flags) ECK(cudaMemcpyAsync(flags, e->d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost, e->stream));
  if (inst_flags)
    ECK(cudaMemcpyAsync(inst_flags, e->d_inst_status, sizeof(uint32_t) * e->ninst, cudaMemcpyDeviceToHost, e->stream));
  ECK(cudaStreamSynchronize(e->stream));
  return 0;
}

int amrvac_ens_set_grid(amrvac_ens *e, int ctas) {
  if (int r = check_ens(e)) return r;
  if (ctas < 0) return efail(AMRVAC_E_ARG, "ctas must be >= 0");
  const int g = ctas == 0 ? e->wave : ctas;
  if (g != e->grid && e->graph) {
    cudaGraphExecDestroy(e->graph);
    e->graph = nullptr;
  }
  e->grid = g;
  return 0;
}

int amrvac_ens_grid(const amrvac_ens *e, int *ctas, int *wave) {
  if (!e) return AMRVAC_E_ARG;
  if (ctas) *ctas = e->grid;
  if (wave) *wave = e->wave;
  return 0;
}

int amrvac_ens_set_variant(amrvac_ens *e, int var) {
  if (int r = check_ens(e)) return r;
  if (var < 0 || var >= e->nvar) return efail(AMRVAC_E_ARG, "no such stage-kernel variant");
  if (var != e->var && e->graph) {
    cudaGraphExecDestroy(e->graph);
    e->graph = nullptr;
  }
  if (e->grid == e->wave) e->grid = e->wave_v[var];  // one resident wave stays one wave
  e->var = var;
  e->wave = e->wave_v[var];
  return 0;
}

int amrvac_ens_variant(const amrvac_ens *e, int *var, int *nvar, int *ctas_per_sm) {
  if (!e) return AMRVAC_E_ARG;
  if (var) *var = e->var;
  if (nvar) *nvar = e->nvar;
  if (ctas_per_sm) *ctas_per_sm = ens_variant_ctas(e->mixed, e->var);  // the launch bounds of the variant
  return 0;
}

// Times one forward-Euler-like stage (register 0 -> 1, the state in 0 is
// untouched) for each stage-kernel variant and candidate grid size, and
// keeps the fastest pair.
int amrvac_ens_autotune(amrvac_ens *e, int reps, int *best_ctas, double *best_ms) {
  if (int r = check_ens(e)) return r;
  if (reps <= 0) reps = 5;
  // dt of the current state, as the stages read it
  const EnsArgs G = ens_args(e, 0, 0, 0, 0.0, 1.0, 1.0);
  ens_getdt_kernel<<<e->grid, STAGE_THREADS, 0, e->stream>>>(G);
  const EnsTime T = ens_time(e);
  std::vector<int> done_save(e->ninst);
  ECK(cudaMemcpyAsync(done_save.data(), e->d_done, sizeof(int) * e->ninst, cudaMemcpyDeviceToHost, e->stream));
  ens_finalize_kernel<<<(e->ninst + 127) / 128, 128, 0, e->stream>>>(T);
  ECK(cudaGetLastError());
  ECK(cudaStreamSynchronize(e->stream));
  cudaEvent_t a, b;
  ECK(cudaEventCreate(&a));
  ECK(cudaEventCreate(&b));
  double best = 1e30;
  int bestg = e->wave, bestv = e->var;
  const int saved = e->grid, saved_var = e->var;
  auto restore = [&]() {
    e->var = saved_var;
    e->wave = e->wave_v[saved_var];
    e->grid = saved;
  };
  for (int v = 0; v < e->nvar; ++v) {
    e->var = v;
    e->wave = e->wave_v[v];
    const int cands[4] = {e->wave, 2 * e->wave, 4 * e->wave, e->wave / 2};
    for (int c : cands) {
      if (c <= 0) continue;
      e->grid = c;
      int r = ens_launch_stage(e, 0, 1, 0, 0.0, 1.0, 1.0);  // warm-up
      if (r) { restore(); return r; }
      ECK(cudaEventRecord(a, e->stream));
      for (int q = 0; q < reps && !r; ++q) r = ens_launch_stage(e, 0, 1, 0, 0.0, 1.0, 1.0);
      ECK(cudaEventRecord(b, e->stream));
      ECK(cudaEventSynchronize(b));
      if (r) { restore(); return r; }
      float ms = 0;
      ECK(cudaEventElapsedTime(&ms, a, b));
      if (ms / reps < best) { best = ms / reps; bestg = c; bestv = v; }
    }
  }
  restore();
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  // the probe must not change the instances' clocks: restore done flags and dt
  ECK(cudaMemcpyAsync(e->d_done, done_save.data(), sizeof(int) * e->ninst, cudaMemcpyHostToDevice, e->stream));
  ECK(cudaMemsetAsync(e->d_dt, 0, sizeof(double) * e->ninst, e->stream));
  ECK(cudaStreamSynchronize(e->stream));
  if (int r = amrvac_ens_set_variant(e, bestv)) return r;
  if (int r = amrvac_ens_set_grid(e, bestg)) return r;
  if (best_ctas) *best_ctas = bestg;
  if (best_ms) *best_ms = best;
  return 0;
}

int amrvac_ens_stream(amrvac_ens *e, void **stream) {
  if (int r = check_ens(e)) return r;
  if (!stream) return efail(AMRVAC_E_ARG, "null argument");
  *stream = e->stream;
  return 0;
}

int64_t amrvac_ens_launch_count(const amrvac_ens *e) { return e ? e->launches : -1; }

}  // extern "C"
