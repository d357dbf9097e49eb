// Fused finite-volume stage kernel for 16^d blocks (d = 2, 3).
//
// One CTA advances one block (or a z-chunk of a 3-D block) by one explicit
// stage.  It restates, for all cells of its tile at once:
//   finite_volume (src/mod_finite_volume.t:116-339): primitives, limited
//     reconstruction (reconstruct_LR 1110-1228), GLM modify_wLR, physical
//     fluxes, signal-speed bounds, Riemann flux, conservative update;
//   the SSP-RK stage combination (src/mod_advance.t:249-267);
//   the unsplit divB sources (add_source_glm / add_source_linde,
//     src/mhd/mod_mhd_phys.t:5472-5531, 5599-5665);
//   the same-resolution ghost fill (bc_fill_srl, src/mod_ghostcells_update.t:
//     812-852) and cont/symm/asymm physical boundaries, done as a gather from
//     the neighbour blocks' interiors while staging the tile.
//
// Layout in HBM: pool[block][var][z][y][x], interior cells only, 16^d per
// block and variable (2 KB rows of 16 doubles).  No ghost cells are stored.
//
// CTA organisation (3-D): 288 threads march over the z-planes of the tile.
// Shared memory holds a ring of 4 primitive planes (k-1..k+2, 16x16 each),
// the x/y halo strips of plane k, and one buffer of scaled face fluxes.
// Per plane: x-faces (17x16 = 272, one per thread), per-cell accumulation,
// y-faces (16x17), accumulation, then each cell thread computes its own
// z-face k+1/2 and keeps the k-1/2 flux in registers.
#pragma once

#include <cuda_runtime.h>

#include "physics.cuh"
#include "riemann.cuh"

namespace amrvac {

constexpr int BN = 16;               // cells per block edge
constexpr int STAGE_THREADS = 288;   // 9 warps: 17*16 faces + 16 spare

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
};

__device__ __forceinline__ int dir_index(int di, int dj, int dk) {
  return (di + 1) + 3 * (dj + 1) + 9 * (dk + 1);
}

// Resolve a cell of block b given local coordinates that may lie up to two
// cells outside the block: physical sides first (clamp for cont, mirror for
// symm/asymm), then the remaining offset through the neighbour table.
template <int NDIM>
__device__ __forceinline__ int resolve_cell(const StageArgs &A, int b, int &i, int &j, int &k,
                                            uint32_t &flip) {
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
    if (nf < 0) {
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
__device__ __forceinline__ size_t cell_offset(int blk, int nw, int v, int i, int j, int k) {
  constexpr int NY = NDIM >= 2 ? BN : 1;
  constexpr int NZ = NDIM >= 3 ? BN : 1;
  return (((size_t)blk * nw + v) * NZ + k) * (size_t)(NY * BN) + (size_t)j * BN + i;
}

// Load the conserved state of a (possibly out-of-block) cell and return it
// as primitives.  Returns a status bit if the small-value check fires.
template <bool MHD, int NDIR, bool GLM, int NDIM>
__device__ __forceinline__ uint32_t load_prim(const StageArgs &A, int b, int i, int j, int k,
                                              double *w) {
  using V = Vars<MHD, NDIR, GLM>;
  uint32_t flip;
  const int blk = resolve_cell<NDIM>(A, b, i, j, k, flip);
#pragma unroll
  for (int v = 0; v < V::NW; ++v) {
    double x = __ldg(A.uin + cell_offset<NDIM>(blk, V::NW, v, i, j, k));
    w[v] = ((flip >> v) & 1u) ? -x : x;
  }
  uint32_t st = 0;
  if (A.P.fix_small_values) {
    if (small_values<MHD, NDIR, GLM>(w, false, A.P) && A.P.small_values_method != 1) st |= ST_SMALL_VALUE;
  }
  to_primitive<MHD, NDIR, GLM>(w, A.P);
  return st;
}

// Interface flux from reconstructed primitive left/right states: small-value
// fix, to_conserved, GLM modify_wLR, physical fluxes, cbounds, Riemann solver
// (src/mod_finite_volume.t:1217-1222, 200-245).  wLp/wRp are modified.
template <bool MHD, int NDIR, bool GLM, int NDIM, int SOLVER, int BS>
__device__ __forceinline__ uint32_t face_from_states(double *wLp, double *wRp, const PhysParams &P,
                                                     double cg, double *F) {
  constexpr int D = 0;  // states arrive rotated: the face normal is component 0
  using V = Vars<MHD, NDIR, GLM>;
  constexpr int NW = V::NW;
  uint32_t st = 0;
  if (P.fix_small_values) {
    bool fl = small_values<MHD, NDIR, GLM>(wLp, true, P);
    bool fr = small_values<MHD, NDIR, GLM>(wRp, true, P);
    if ((fl || fr) && P.small_values_method != 1) st |= ST_SMALL_VALUE;
  }
  double wLC[NW], wRC[NW];
#pragma unroll
  for (int v = 0; v < NW; ++v) { wLC[v] = wLp[v]; wRC[v] = wRp[v]; }
  to_conserved<MHD, NDIR, GLM>(wLC, P);
  to_conserved<MHD, NDIR, GLM>(wRC, P);
  if constexpr (MHD && GLM) {
    // mhd_modify_wLR (src/mhd/mod_mhd_phys.t:6352-6372)
    constexpr int BNI = V::B0 + D, PS = V::PSI, E = V::E;
    const double dB = wRp[BNI] - wLp[BNI];
    const double dPsi = wRp[PS] - wLp[PS];
    const double nb = 0.5 * (wRp[BNI] + wLp[BNI] - dPsi / cg);
    const double np = 0.5 * (wRp[PS] + wLp[PS] - dB * cg);
    wLp[BNI] = nb; wLp[PS] = np; wRp[BNI] = nb; wRp[PS] = np;
    wRC[E] = wRC[E] - 0.5 * (wRC[BNI] * wRC[BNI]);
    wLC[E] = wLC[E] - 0.5 * (wLC[BNI] * wLC[BNI]);
    wRC[BNI] = nb; wRC[PS] = np; wLC[BNI] = nb; wLC[PS] = np;
    wRC[E] = wRC[E] + 0.5 * (nb * nb);
    wLC[E] = wLC[E] + 0.5 * (nb * nb);
  }
  double fL[NW], fR[NW];
  phys_flux<MHD, NDIR, GLM, D>(wLC, wLp, cg, fL);
  phys_flux<MHD, NDIR, GLM, D>(wRC, wRp, cg, fR);
  double cmax, cmin = 0.0;
  if constexpr (SOLVER == SOLVER_TVDLF) {
    st |= cbounds<MHD, NDIR, GLM, D, false, BS>(wLC, wRC, wLp, wRp, P, cmax, cmin);
    riemann_tvdlf<NW>(wLC, wRC, fL, fR, cmax, P.tvdlfeps, F);
  } else {
    st |= cbounds<MHD, NDIR, GLM, D, true, BS>(wLC, wRC, wLp, wRp, P, cmax, cmin);
    if constexpr (SOLVER == SOLVER_HLL) {
      riemann_hll<MHD, NDIR, GLM, NDIM, D>(wLC, wRC, fL, fR, cmax, cmin, P.tvdlfeps, F);
    } else if constexpr (SOLVER == SOLVER_HLLC) {
      static_assert(!MHD, "HLLC is implemented for HD only");
      riemann_hllc_hd<NDIR, D>(wLC, wRC, fL, fR, cmax, cmin, F);
    } else {
      static_assert(MHD, "HLLD needs MHD");
      riemann_hlld<NDIR, GLM, NDIM, D>(wLC, wRC, wLp, wRp, fL, fR, cmax, cmin, F);
    }
  }
  return st;
}

// One face normal to direction D: primitives of the 4-cell stencil (cells
// L-1, L, R, R+1) are read through `ld(o, v)` with o in {-2,-1,0,1} relative
// to the right cell and v in the reference variable order.  The states are
// rotated so that one direction-generic face routine serves x, y and z; the
// flux F is returned in the reference order.
template <bool MHD, int NDIR, bool GLM, int NDIM, int SOLVER, int LIM, int BS, int D, class LD>
__device__ __forceinline__ uint32_t face_flux(const LD &ld, const PhysParams &P, double cg,
                                              double rdelinv, double *F) {
  using V = Vars<MHD, NDIR, GLM>;
  constexpr int NW = V::NW;
  double wLp[NW], wRp[NW];
#pragma unroll
  for (int v = 0; v < NW; ++v) {
    const int ov = orig_index<MHD, NDIR, D>(v);
    const double q0 = ld(-2, ov), q1 = ld(-1, ov), q2 = ld(0, ov), q3 = ld(1, ov);
    const double d0 = q1 - q0, d1 = q2 - q1, d2 = q3 - q2;
    wLp[v] = q1 + 0.5 * limited_slope<true, LIM>(P.limiter, d1, d0, rdelinv);
    wRp[v] = q2 - 0.5 * limited_slope<false, LIM>(P.limiter, d2, d1, rdelinv);
  }
  double Fr[NW];
  const uint32_t st = face_from_states<MHD, NDIR, GLM, NDIM, SOLVER, BS>(wLp, wRp, P, cg, Fr);
#pragma unroll
  for (int v = 0; v < NW; ++v) F[orig_index<MHD, NDIR, D>(v)] = Fr[v];
  return st;
}

// Shared-memory tile (sizes in doubles).
template <int NW, int NDIM>
struct Tile {
  static constexpr int NSLOT = NDIM == 3 ? 4 : 1;
  static constexpr int PLANE = BN * BN;
  static constexpr int RING = NSLOT * NW * PLANE;        // [slot][v][j][i]
  static constexpr int HX = NW * BN * 4;                 // [v][j][c] c: i=-2,-1,16,17
  static constexpr int HY = NW * 4 * BN;                 // [v][r][i] r: j=-2,-1,16,17
  static constexpr int HC = NW * 16;                     // [v][r][c] corners
  static constexpr int FB = NW * (BN + 1) * BN;          // [v][face]
  static constexpr int TOTAL = RING + HX + HY + HC + FB;
  static constexpr size_t BYTES = sizeof(double) * TOTAL;
};

__device__ __forceinline__ int halo_slot(int c) { return c < 0 ? c + 2 : c - (BN - 2); }

template <int NW, int NDIM>
struct TileView {
  double *ring, *hx, *hy, *hc, *fb;
  __device__ TileView(double *s) {
    using T = Tile<NW, NDIM>;
    ring = s;
    hx = ring + T::RING;
    hy = hx + T::HX;
    hc = hy + T::HY;
    fb = hc + T::HC;
  }
  // primitive v at in-plane (i, j) in [-2, 17]^2 of the plane held in `slot`
  __device__ __forceinline__ double at(int slot, int v, int i, int j) const {
    const bool ii = (unsigned)i < (unsigned)BN, jj = (unsigned)j < (unsigned)BN;
    if (ii && jj) return ring[(slot * NW + v) * (BN * BN) + j * BN + i];
    if (jj) return hx[(v * BN + j) * 4 + halo_slot(i)];
    if (ii) return hy[(v * 4 + halo_slot(j)) * BN + i];
    return hc[(v * 4 + halo_slot(j)) * 4 + halo_slot(i)];
  }
  __device__ __forceinline__ double &center(int slot, int v, int i, int j) {
    return ring[(slot * NW + v) * (BN * BN) + j * BN + i];
  }
};

template <bool MHD, int NDIR, bool GLM, int NDIM, int SOLVER, int LIM, int BS>
__global__ void __launch_bounds__(STAGE_THREADS, 1) fv_stage_kernel(const StageArgs A) {
  using V = Vars<MHD, NDIR, GLM>;
  constexpr int NW = V::NW;
  extern __shared__ double smem[];
  TileView<NW, NDIM> tv(smem);
  const int t = threadIdx.x;
  const int nchunk = NDIM == 3 ? BN / A.zchunk : 1;
  const int b = blockIdx.x / nchunk;
  const int chunk = blockIdx.x - b * nchunk;
  const int k0 = NDIM == 3 ? chunk * A.zchunk : 0;
  const int k1 = NDIM == 3 ? k0 + A.zchunk : 1;
  if (b >= A.nblocks) return;

  const PhysParams &P = A.P;
  const double dt = *A.dt_dev;
  const double qdt = A.dtfactor * dt;
  const double cg = GLM ? *A.cmax_dev : 0.0;
  double dx[3], dxinv[3], rdel[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    dx[d] = d < NDIM ? A.dxb[b * 3 + d] : 1.0;
    dxinv[d] = -qdt / dx[d];
    const double r = P.cada3_radius * dx[d];
    rdel[d] = 1.0 / (r * r);
  }
  uint32_t st = 0;
  const int ci = t & (BN - 1), cj = t >> 4;  // cell role for t < 256
  const bool cell_thread = t < BN * BN;
  const bool need_corners = MHD && !GLM && P.divb == DIVB_LINDE;

  auto load_center = [&](int kk) {
    if (cell_thread) {
      double w[NW];
      st |= load_prim<MHD, NDIR, GLM, NDIM>(A, b, ci, cj, kk, w);
      const int slot = NDIM == 3 ? (kk & 3) : 0;
#pragma unroll
      for (int v = 0; v < NW; ++v) tv.center(slot, v, ci, cj) = w[v];
    }
  };
  auto load_halo = [&](int kk) {
    // x strips: 64 cells, y strips: 64 cells, corners: 16 cells
    const int ncell = need_corners ? 144 : 128;
    for (int h = t; h < ncell; h += STAGE_THREADS) {
      int i, j;
      double *dst;
      int stride;
      if (h < 64) {
        j = h >> 2;
        const int c = h & 3;
        i = c < 2 ? c - 2 : c + BN - 2;
        dst = tv.hx + j * 4 + c;
        stride = BN * 4;
      } else if (h < 128) {
        const int r = (h - 64) >> 4;
        i = (h - 64) & (BN - 1);
        j = r < 2 ? r - 2 : r + BN - 2;
        dst = tv.hy + r * BN + i;
        stride = 4 * BN;
      } else {
        const int r = (h - 128) >> 2, c = (h - 128) & 3;
        i = c < 2 ? c - 2 : c + BN - 2;
        j = r < 2 ? r - 2 : r + BN - 2;
        dst = tv.hc + r * 4 + c;
        stride = 16;
      }
      double w[NW];
      st |= load_prim<MHD, NDIR, GLM, NDIM>(A, b, i, j, kk, w);
#pragma unroll
      for (int v = 0; v < NW; ++v) dst[v * stride] = w[v];
    }
  };

  // z-face k+1/2 for the column of this cell thread, from ring planes k-1..k+2
  auto zface = [&](int k, double *Fs) {
    if constexpr (NDIM == 3) {
      auto ld = [&](int o, int v) -> double {
        return tv.ring[(((k + 1 + o) & 3) * NW + v) * (BN * BN) + cj * BN + ci];
      };
      st |= face_flux<MHD, NDIR, GLM, NDIM, SOLVER, LIM, BS, 2>(ld, P, cg, rdel[2], Fs);
#pragma unroll
      for (int v = 0; v < NW; ++v) Fs[v] = dxinv[2] * Fs[v];
    }
  };

  double fz_prev[NDIM == 3 ? NW : 1];
  if constexpr (NDIM == 3) {
    load_center(k0 - 2);
    load_center(k0 - 1);
    load_center(k0);
    load_center(k0 + 1);
    __syncthreads();
    if (cell_thread) zface(k0 - 1, fz_prev);
    __syncthreads();  // the first iteration overwrites ring slot (k0-2)&3
  }

  for (int k = k0; k < k1; ++k) {
    const int slot = NDIM == 3 ? (k & 3) : 0;
    if constexpr (NDIM == 3) load_center(k + 2);
    else load_center(0);
    load_halo(k);
    // RK combination wnew0 = a*base + b*in (src/mod_advance.t:254-266)
    double acc[NW];
    if (cell_thread) {
#pragma unroll
      for (int v = 0; v < NW; ++v) {
        const size_t o = cell_offset<NDIM>(b, NW, v, ci, cj, k);
        const double win = A.uin[o];
        acc[v] = (A.a_base == 0.0) ? win : A.a_base * A.ubase[o] + A.b_in * win;
      }
    }
    __syncthreads();
    // ---- x faces: face (fi - 1/2) of row fj, fi in [0,16]
    if (t < (BN + 1) * BN) {
      const int fj = t / (BN + 1), fi = t - fj * (BN + 1);
      auto ld = [&](int o, int v) -> double { return tv.at(slot, v, fi + o, fj); };
      double F[NW];
      st |= face_flux<MHD, NDIR, GLM, NDIM, SOLVER, LIM, BS, 0>(ld, P, cg, rdel[0], F);
#pragma unroll
      for (int v = 0; v < NW; ++v) tv.fb[v * ((BN + 1) * BN) + t] = dxinv[0] * F[v];
    }
    __syncthreads();
    if (cell_thread) {
      const int f = cj * (BN + 1) + ci;
#pragma unroll
      for (int v = 0; v < NW; ++v) {
        const double *fb = tv.fb + v * ((BN + 1) * BN);
        acc[v] = acc[v] + fb[f + 1] - fb[f];
      }
    }
    __syncthreads();
    // ---- y faces: face (fj - 1/2) of column fi, fj in [0,16]
    if (t < (BN + 1) * BN) {
      const int fj = t >> 4, fi = t & (BN - 1);
      auto ld = [&](int o, int v) -> double { return tv.at(slot, v, fi, fj + o); };
      double F[NW];
      st |= face_flux<MHD, NDIR, GLM, NDIM, SOLVER, LIM, BS, 1>(ld, P, cg, rdel[1], F);
#pragma unroll
      for (int v = 0; v < NW; ++v) tv.fb[v * ((BN + 1) * BN) + t] = dxinv[1] * F[v];
    }
    __syncthreads();
    if (cell_thread) {
      const int f = cj * BN + ci;
#pragma unroll
      for (int v = 0; v < NW; ++v) {
        const double *fb = tv.fb + v * ((BN + 1) * BN);
        acc[v] = acc[v] + fb[f + BN] - fb[f];
      }
      // ---- z face k+1/2 (registers)
      if constexpr (NDIM == 3) {
        double fz[NW];
        zface(k, fz);
#pragma unroll
        for (int v = 0; v < NW; ++v) {
          acc[v] = acc[v] + fz[v] - fz_prev[v];
          fz_prev[v] = fz[v];
        }
      }
      // ---- small values on wnew (src/mod_finite_volume.t:326-333)
      if (P.fix_small_values) {
        if (small_values<MHD, NDIR, GLM>(acc, false, P) && P.small_values_method != 1) {
          st |= ST_SMALL_VALUE;
          atomicOr(A.block_status + b, ST_SMALL_VALUE);
        }
      }
      // ---- unsplit divB sources (addsource2 -> mhd_add_source)
      if constexpr (MHD) {
        if (NDIM > 1) {
          const double qsrc = qdt * double(NDIM) / double(NDIM);
          if constexpr (GLM) {
            // add_source_glm (src/mhd/mod_mhd_phys.t:5472-5531)
            double mindx = dx[0];
#pragma unroll
            for (int d = 1; d < NDIM; ++d) mindx = fmin(mindx, dx[d]);
            if (P.glm_alpha < 0.0) {
              acc[V::PSI] = fabs(P.glm_alpha) * A.uin[cell_offset<NDIM>(b, NW, V::PSI, ci, cj, k)];
            } else {
              acc[V::PSI] = exp(-(qsrc * cg * P.glm_alpha) / mindx) * acc[V::PSI];
            }
            if (P.glm_extended) {
              auto nbv = [&](int d, int s, int v) -> double {  // wCT at cell +/- e_d
                if (d == 0) return tv.at(slot, v, ci + s, cj);
                if (d == 1) return tv.at(slot, v, ci, cj + s);
                return tv.ring[((((k + s) & 3)) * NW + v) * (BN * BN) + cj * BN + ci];
              };
#pragma unroll
              for (int d = 0; d < NDIM; ++d) {
                const double g = ((nbv(d, 1, V::PSI) - nbv(d, -1, V::PSI)) * 0.5) / dx[d];
                acc[V::E] = acc[V::E] - qsrc * tv.at(slot, V::B0 + d, ci, cj) * g;
              }
              double divb = 0.0;
#pragma unroll
              for (int d = 0; d < NDIM; ++d)
                divb = divb + 0.5 * (nbv(d, 1, V::B0 + d) - nbv(d, -1, V::B0 + d)) * (1.0 / dx[d]);
#pragma unroll
              for (int c = 0; c < NDIR; ++c)
                acc[V::M0 + c] = acc[V::M0 + c] - qsrc * tv.at(slot, V::B0 + c, ci, cj) * divb;
            }
          } else if (P.divb == DIVB_LINDE) {
            if constexpr (NDIM == 2) {
              // add_source_linde (src/mhd/mod_mhd_phys.t:5599-5665), uniform grid
              auto divb_at = [&](int i, int j) -> double {
                double d = 0.5 * (tv.at(slot, V::B0, i + 1, j) - tv.at(slot, V::B0, i - 1, j)) * (1.0 / dx[0]);
                d = d + 0.5 * (tv.at(slot, V::B0 + 1, i, j + 1) - tv.at(slot, V::B0 + 1, i, j - 1)) * (1.0 / dx[1]);
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
                acc[V::E] = acc[V::E] + tv.at(slot, V::B0 + d, ci, cj) * g;
              }
            }
          }
          if (P.fix_small_values) {
            if (small_values<MHD, NDIR, GLM>(acc, false, P) && P.small_values_method != 1) st |= ST_SMALL_VALUE;
          }
        }
      }
#pragma unroll
      for (int v = 0; v < NW; ++v) A.uout[cell_offset<NDIM>(b, NW, v, ci, cj, k)] = acc[v];
    }
    __syncthreads();
  }
  if (st) atomicOr(A.status, st);
}

}  // namespace amrvac
