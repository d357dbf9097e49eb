// Device side of the AMR decisions: the Löhner error estimator
// (lohner_grid, src/amr/mod_errest.t:63-200, refine_criterion 3) on the
// resident blocks, feeding the host's regrid with one flag per block instead
// of the whole state.
//
// Per interior cell and weighted variable (optionally log10):
//   numerator   = sum_d sum_d2 (t_d(c+e_d2) - t_d(c-e_d2))^2,
//                 t_d(p) = w(p+e_d) - w(p-e_d)
//   denominator = sum_d sum_d2 (|w(c+2e_d)-w(c)| + |w(c)-w(c-2e_d)|
//                               + wavefilter (a_d(c+e_d2) + a_d(c-e_d2)))^2,
//                 a_d(p) = |w(p+e_d)| + |w(p-e_d)|
//   error      += weight sqrt(numerator / max(denominator, 1e-6))
// in the reference's operation order; the block is flagged for refinement if
// any cell has error >= threshold(level) (and level < refine_max_level), for
// coarsening if every cell has error <= derefine_ratio(level) threshold(level)
// (and level > 1).  The 19-point stencil (axial +-2, face-diagonal +-1) is
// read through the same neighbour-table gather as the stage kernel, so ghost
// values are those getbc would produce.
#include "amr.cuh"

namespace amrvac {

namespace {

template <int NDIM>
__global__ void __launch_bounds__(256) lohner_kernel(const LohnerArgs A) {
  const int b = blockIdx.x;
  const int t = threadIdx.x;
  const StageArgs &S = A.sa;
  const int bn = S.bn;
  const int nw = A.nw;
  const int lev = A.level[b];
  const double wf = A.wavefilter[lev - 1], thr = A.threshold[lev - 1], der = A.derefine[lev - 1];
  auto wv = [&](int iw, int x, int y, int z) -> double {
    int ii = x, jj = y, kk = z;
    uint32_t flip;
    const int blk = resolve_cell<NDIM>(S, b, ii, jj, kk, flip, bn);
    // a level jump (blk <= -2) reads the ghost buffer the ghost pass filled
    double v = blk >= 0 ? S.uin[cell_offset<NDIM>(blk, nw, iw, ii, jj, kk, bn)]
                        : S.gbuf[ghost_offset<NDIM>(-2 - blk, nw, iw, ii, jj, kk, bn)];
    if ((flip >> iw) & 1u) v = -v;
    return ((A.logflag >> iw) & 1u) ? log10(v) : v;
  };
  bool any_ref = false, all_coa = true;
  double emax = 0.0;
  const int ncell = bn * (NDIM >= 2 ? bn : 1) * (NDIM == 3 ? bn : 1);
  for (int cell = t; cell < ncell; cell += 256) {  // the block's cells, x fastest
    const int i = cell % bn, j = NDIM >= 2 ? (cell / bn) % bn : 0, k = NDIM == 3 ? cell / (bn * bn) : 0;
    double err = 0.0;
    for (int iw = 0; iw < nw; ++iw) {
      const double wt = A.weight[iw];
      if (wt == 0.0) continue;
      double num = 0.0, den = 0.0;
#pragma unroll
      for (int d = 0; d < NDIM; ++d) {
        const int e0 = d == 0, e1 = d == 1, e2 = d == 2;
#pragma unroll
        for (int d2 = 0; d2 < NDIM; ++d2) {
          const int f0 = d2 == 0, f1 = d2 == 1, f2 = d2 == 2;
          // t_d(c+f) - t_d(c-f)
          const double tp = wv(iw, i + f0 + e0, j + f1 + e1, k + f2 + e2) - wv(iw, i + f0 - e0, j + f1 - e1, k + f2 - e2);
          const double tm = wv(iw, i - f0 + e0, j - f1 + e1, k - f2 + e2) - wv(iw, i - f0 - e0, j - f1 - e1, k - f2 - e2);
          const double q = tp - tm;
          num = num + q * q;
        }
      }
#pragma unroll
      for (int d = 0; d < NDIM; ++d) {
        const int e0 = d == 0, e1 = d == 1, e2 = d == 2;
        const double c = wv(iw, i, j, k);
        const double ta = fabs(wv(iw, i + 2 * e0, j + 2 * e1, k + 2 * e2) - c) +
                          fabs(c - wv(iw, i - 2 * e0, j - 2 * e1, k - 2 * e2));
#pragma unroll
        for (int d2 = 0; d2 < NDIM; ++d2) {
          const int f0 = d2 == 0, f1 = d2 == 1, f2 = d2 == 2;
          const double ap = fabs(wv(iw, i + f0 + e0, j + f1 + e1, k + f2 + e2)) +
                            fabs(wv(iw, i + f0 - e0, j + f1 - e1, k + f2 - e2));
          const double am = fabs(wv(iw, i - f0 + e0, j - f1 + e1, k - f2 + e2)) +
                            fabs(wv(iw, i - f0 - e0, j - f1 - e1, k - f2 - e2));
          const double q = ta + wf * (ap + am);
          den = den + q * q;
        }
      }
      err = err + wt * sqrt(num / fmax(den, 1.0e-6));
    }
    if (err >= thr) { any_ref = true; all_coa = false; }
    else if (!(err <= der * thr)) all_coa = false;
    emax = fmax(emax, err);
  }
  // block reduction
  __shared__ double red[8];
  const int r_any = __syncthreads_or(any_ref);
  const int r_all = __syncthreads_and(all_coa);
  double m = emax;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((t & 31) == 0) red[t >> 5] = m;
  __syncthreads();
  if (t == 0) {
    double mm = 0.0;
    for (int q = 0; q < 8; ++q) mm = fmax(mm, red[q]);
    int fl = 0;
    if (r_any && lev < A.refine_max_level) fl |= 1;
    if (r_all && lev > 1) fl |= 2;
    A.flags[b] = fl;
    A.errmax[b] = mm;
  }
}

// The same estimator with each weighted variable's ghosted block (two
// layers, the cells the stencil reaches) gathered once into shared memory —
// the same gather, flips and log10 as lohner_kernel's wv — and the stencils
// read from there; per-cell error sums in shared memory, variables in
// ascending order as there.
template <int NDIM>
__global__ void __launch_bounds__(256) lohner_staged_kernel(const LohnerArgs A) {
  extern __shared__ double lsm[];
  const int b = blockIdx.x;
  const int t = threadIdx.x;
  const StageArgs &S = A.sa;
  const int bn = S.bn;
  const int nw = A.nw;
  const int lev = A.level[b];
  const double wf = A.wavefilter[lev - 1], thr = A.threshold[lev - 1], der = A.derefine[lev - 1];
  const int G = bn + 4, GY = NDIM >= 2 ? G : 1, GZ = NDIM == 3 ? G : 1;
  const int ng = G * GY * GZ;
  const int ncell = bn * (NDIM >= 2 ? bn : 1) * (NDIM == 3 ? bn : 1);
  double *sw = lsm, *serr = lsm + ng;
  for (int cell = t; cell < ncell; cell += 256) serr[cell] = 0.0;
  // staged value at block-local (x, y, z), each in -2 .. bn+1
  auto at = [&](int x, int y, int z) -> double {
    return sw[(x + 2) + G * ((NDIM >= 2 ? y + 2 : 0) + GY * (NDIM == 3 ? z + 2 : 0))];
  };
  for (int iw = 0; iw < nw; ++iw) {
    const double wt = A.weight[iw];
    if (wt == 0.0) continue;
    __syncthreads();  // the previous variable's stencils are read
    for (int p = t; p < ng; p += 256) {
      const int x = p % G - 2, y = NDIM >= 2 ? (p / G) % GY - 2 : 0, z = NDIM == 3 ? p / (G * GY) - 2 : 0;
      // reached by the stencil: +-2 along one axis, or +-1 along two
      const int ox = x < 0 ? -x : (x >= bn ? x - bn + 1 : 0);
      const int oy = y < 0 ? -y : (y >= bn ? y - bn + 1 : 0);
      const int oz = z < 0 ? -z : (z >= bn ? z - bn + 1 : 0);
      const int nout = (ox > 0) + (oy > 0) + (oz > 0);
      if (nout > 2 || (nout == 2 && (ox > 1 || oy > 1 || oz > 1))) continue;
      int ii = x, jj = y, kk = z;
      uint32_t flip;
      const int blk = resolve_cell<NDIM>(S, b, ii, jj, kk, flip, bn);
      double v = blk >= 0 ? S.uin[cell_offset<NDIM>(blk, nw, iw, ii, jj, kk, bn)]
                          : S.gbuf[ghost_offset<NDIM>(-2 - blk, nw, iw, ii, jj, kk, bn)];
      if ((flip >> iw) & 1u) v = -v;
      sw[p] = ((A.logflag >> iw) & 1u) ? log10(v) : v;
    }
    __syncthreads();
    for (int cell = t; cell < ncell; cell += 256) {
      const int i = cell % bn, j = NDIM >= 2 ? (cell / bn) % bn : 0, k = NDIM == 3 ? cell / (bn * bn) : 0;
      double num = 0.0, den = 0.0;
#pragma unroll
      for (int d = 0; d < NDIM; ++d) {
        const int e0 = d == 0, e1 = d == 1, e2 = d == 2;
#pragma unroll
        for (int d2 = 0; d2 < NDIM; ++d2) {
          const int f0 = d2 == 0, f1 = d2 == 1, f2 = d2 == 2;
          const double tp = at(i + f0 + e0, j + f1 + e1, k + f2 + e2) - at(i + f0 - e0, j + f1 - e1, k + f2 - e2);
          const double tm = at(i - f0 + e0, j - f1 + e1, k - f2 + e2) - at(i - f0 - e0, j - f1 - e1, k - f2 - e2);
          const double q = tp - tm;
          num = num + q * q;
        }
      }
#pragma unroll
      for (int d = 0; d < NDIM; ++d) {
        const int e0 = d == 0, e1 = d == 1, e2 = d == 2;
        const double c = at(i, j, k);
        const double ta = fabs(at(i + 2 * e0, j + 2 * e1, k + 2 * e2) - c) +
                          fabs(c - at(i - 2 * e0, j - 2 * e1, k - 2 * e2));
#pragma unroll
        for (int d2 = 0; d2 < NDIM; ++d2) {
          const int f0 = d2 == 0, f1 = d2 == 1, f2 = d2 == 2;
          const double ap = fabs(at(i + f0 + e0, j + f1 + e1, k + f2 + e2)) +
                            fabs(at(i + f0 - e0, j + f1 - e1, k + f2 - e2));
          const double am = fabs(at(i - f0 + e0, j - f1 + e1, k - f2 + e2)) +
                            fabs(at(i - f0 - e0, j - f1 - e1, k - f2 - e2));
          const double q = ta + wf * (ap + am);
          den = den + q * q;
        }
      }
      serr[cell] = serr[cell] + wt * sqrt(num / fmax(den, 1.0e-6));
    }
  }
  __syncthreads();
  bool any_ref = false, all_coa = true;
  double emax = 0.0;
  for (int cell = t; cell < ncell; cell += 256) {
    const double err = serr[cell];
    if (err >= thr) { any_ref = true; all_coa = false; }
    else if (!(err <= der * thr)) all_coa = false;
    emax = fmax(emax, err);
  }
  __shared__ double red[8];
  const int r_any = __syncthreads_or(any_ref);
  const int r_all = __syncthreads_and(all_coa);
  double m = emax;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((t & 31) == 0) red[t >> 5] = m;
  __syncthreads();
  if (t == 0) {
    double mm = 0.0;
    for (int q = 0; q < 8; ++q) mm = fmax(mm, red[q]);
    int fl = 0;
    if (r_any && lev < A.refine_max_level) fl |= 1;
    if (r_all && lev > 1) fl |= 2;
    A.flags[b] = fl;
    A.errmax[b] = mm;
  }
}

}  // namespace

// ---------------------------------------------------------------- level jumps
// The ghost values of the reference's multi-level getbc
// (src/mod_ghostcells_update.t:350-578) are all coarse-level data at an
// absolute index: a leaf's interior cell where a leaf of that level covers
// it, or the average of the 2^d cells of the finer leaf that refines it
// (coarsen_grid, src/amr/mod_coarsen.t:12-79, conserved variables).  The
// restricted ghost cells of a coarse block are that average; the coarse
// representation psc of a fine block (its own coarsened cells plus the coarse
// neighbours' cells, bc_fill_prolong) is coarse-level data around its
// footprint, from which interpolation_linear (1381-1525) prolongs the fine
// ghost cells with monotonized-central slopes.
// Where a coarse value comes from: the cell itself (n = 1) or its 2^NDIM
// children one level finer (n = 2^NDIM, averaged x fastest), as the address
// of variable 0 (each variable bn^NDIM further); flip: bit v, variable v
// changes sign across a mirror side.  w == nullptr: not found.
struct CoarseSrc {
  const double *w;
  int n;
  uint32_t flip;
};

template <int NDIM>
__device__ CoarseSrc coarse_source(const AmrGhostArgs &A, int L, int P0, int P1, int P2) {
  const int P[3] = {P0, P1, P2};
  int jg[3] = {0, 0, 0}, loc[3] = {0, 0, 0};
  uint32_t flip = 0;
  const int bn = A.bn, half = bn / 2;
#pragma unroll
  for (int d = 0; d < NDIM; ++d) {
    const int n = A.nlev[L][d] * bn;
    int p = P[d];  // within 4 cells of the block and n >= 4: one wrap or mirror
    if (p < 0 || p >= n) {
      // across the domain boundary: the boundary rule at this level, as the
      // coarse neighbour's own physical ghost cells hold it (bc_phys)
      const int side = p < 0 ? 0 : 1;
      const int kind = A.bc_kind[2 * d + side];
      if (kind == BCK_PERIODIC) {
        p = side ? p - n : p + n;
      } else if (kind == BCK_CONT) {
        p = side ? n - 1 : 0;
      } else {
        p = side ? 2 * n - 1 - p : -1 - p;
        flip ^= A.bc_flip[2 * d + side];
      }
    }
    jg[d] = p / bn;
    loc[d] = p - jg[d] * bn;
  }
  const int o = A.owner[A.owner_off[L] + jg[0] + A.nlev[L][0] * (jg[1] + A.nlev[L][1] * jg[2])];
  if (o >= 0) return CoarseSrc{A.u + cell_offset<NDIM>(o, A.nw, 0, loc[0], loc[1], loc[2], bn), 1, flip};
  if (o == -2 && L < A.maxlevel) {
    int jf[3] = {0, 0, 0}, f[3] = {0, 0, 0};
#pragma unroll
    for (int d = 0; d < NDIM; ++d) {
      const int c = loc[d] >= half;
      jf[d] = 2 * jg[d] + c;
      f[d] = 2 * (loc[d] - half * c);
    }
    const int o2 = A.owner[A.owner_off[L + 1] + jf[0] + A.nlev[L + 1][0] * (jf[1] + A.nlev[L + 1][1] * jf[2])];
    if (o2 >= 0)
      return CoarseSrc{A.u + cell_offset<NDIM>(o2, A.nw, 0, f[0], f[1], f[2], bn), 1 << NDIM, flip};
  }
  atomicOr(A.status, ST_BOUNDS);  // hierarchy not 2:1 balanced here
  return CoarseSrc{nullptr, 0, 0u};
}

// Variable v of a coarse value (coarse_source).
template <int NDIM>
__device__ __forceinline__ double coarse_read(const CoarseSrc &s, int v, int bn) {
  if (!s.w) return 0.0;
  const int SY = bn, SZ = bn * bn;
  const double sg = ((s.flip >> v) & 1u) ? -1.0 : 1.0;
  const double *w = s.w + (size_t)v * (NDIM == 3 ? bn * SZ : (NDIM == 2 ? SZ : bn));
  if (s.n == 1) return sg * w[0];
  double sum = w[0];  // x fastest, left to right
  sum = sum + w[1];
  if constexpr (NDIM > 1) {
    sum = sum + w[SY];
    sum = sum + w[SY + 1];
  }
  if constexpr (NDIM > 2) {
    sum = sum + w[SZ];
    sum = sum + w[SZ + 1];
    sum = sum + w[SZ + SY];
    sum = sum + w[SZ + SY + 1];
  }
  return sg * (sum * (1.0 / double(1 << NDIM)));
}

// One CTA per (block next to a level jump, group of AMR_GHOST_VG variables).
// The ghost cells of the level-jump directions are enumerated region by
// region (a face region is 2 x 16 x 16 cells, an edge 2 x 2 x 16, a corner
// 2 x 2 x 2), so no thread walks the interior; the coarse representation psc
// is built first, only where some prolongation stencil reads it.  A thread
// locates a source cell once (coarse_source) and reads it for every variable
// of the group: independent loads in flight together.
// BNC: the block edge as a constant (16, the default) so that the index
// arithmetic folds, or 0 to read it from the arguments.
template <int NDIM, int BNC = 0>
__global__ void __launch_bounds__(256) amr_ghost_kernel(const AmrGhostArgs A) {
  extern __shared__ double psc[];  // [var of the group][(bn/2+4)^NDIM] coarse representation
  const int bn = BNC ? BNC : A.bn;
  const int C = bn / 2 + 4, CY = NDIM >= 2 ? C : 1, CZ = NDIM >= 3 ? C : 1;
  const int CC = C * CY * CZ;
  __shared__ int s_off[28];        // prefix sums of the jump regions' cell counts
  __shared__ int s_q[27], s_kind[27];
  __shared__ int s_nreg;
  __shared__ uint32_t s_coarse;    // bit q: direction q has a coarser neighbour
  __shared__ int s_nt[27];         // the block's neighbour types, loaded by 27 threads at once
  const int slot = blockIdx.x;
  const int v0 = blockIdx.y * AMR_GHOST_VG;
  const int nv = min(AMR_GHOST_VG, A.nw - v0);
  const int b = A.iblocks[slot];
  const int t = threadIdx.x;
  const int L = A.level[b];
  if (t < 27) s_nt[t] = A.ntype[b * 27 + t];
  __syncthreads();
  if (t == 0) {
    const int *nt = s_nt;
    int n = 0, m = 0;
    uint32_t cm = 0;
    for (int q = 0; q < 27; ++q) {
      const int kind = nt[q];
      if (q == 13 || (kind != AMR_COARSE && kind != AMR_FINE)) continue;
      const int dd[3] = {q % 3 - 1, (q / 3) % 3 - 1, q / 9 - 1};
      int cells = 1;
      for (int d = 0; d < NDIM; ++d) cells *= dd[d] ? 2 : bn;
      if (kind == AMR_COARSE) cm |= 1u << q;
      s_q[m] = q;
      s_kind[m] = kind;
      s_off[m] = n;
      n += cells;
      ++m;
    }
    s_off[m] = n;
    s_nreg = m;
    s_coarse = cm;
  }
  __syncthreads();
  const int nreg = s_nreg;
  const uint32_t cmask = s_coarse;
  int igb[3] = {0, 0, 0};
#pragma unroll
  for (int d = 0; d < NDIM; ++d) igb[d] = A.ig[3 * b + d];
  if (cmask) {
    for (int p = t; p < CC; p += blockDim.x) {
      const int pc[3] = {p % C, NDIM >= 2 ? (p / C) % CY : 0, NDIM >= 3 ? p / (C * CY) : 0};
      // read by the stencils (centre +- 1 per direction) of the ghost cells
      // of a coarser-neighbour direction: coarse index 1 for the low ghosts,
      // 2..bn/2+1 beside the block, bn/2+2 for the high ghosts
      // (bit q of kDirBits[d][k + 1]: component d of direction q is k)
      constexpr uint32_t kDirBits[3][3] = {{0x1249249u, 0x2492492u, 0x4924924u},
                                           {0x01c0e07u, 0x0e07038u, 0x70381c0u},
                                           {0x00001ffu, 0x003fe00u, 0x7fc0000u}};
      uint32_t m = cmask;
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        uint32_t md = 0;
        if (d < NDIM) {
          if (pc[d] <= 2) md |= kDirBits[d][0];
          if (pc[d] >= 1 && pc[d] <= bn / 2 + 2) md |= kDirBits[d][1];
          if (pc[d] >= bn / 2 + 1) md |= kDirBits[d][2];
        } else {
          md = kDirBits[d][1];
        }
        m &= md;
      }
      if (!m) continue;
      int P[3] = {0, 0, 0};
#pragma unroll
      for (int d = 0; d < NDIM; ++d) P[d] = igb[d] * (bn / 2) + pc[d] - 2;
      const CoarseSrc src = coarse_source<NDIM>(A, L - 1, P[0], P[1], P[2]);
      double val[AMR_GHOST_VG];
#pragma unroll
      for (int vv = 0; vv < AMR_GHOST_VG; ++vv)
        if (vv < nv) val[vv] = coarse_read<NDIM>(src, v0 + vv, bn);
#pragma unroll
      for (int vv = 0; vv < AMR_GHOST_VG; ++vv)
        if (vv < nv) psc[vv * CC + p] = val[vv];
    }
    __syncthreads();
  }
  double dxF[3] = {1, 1, 1}, dxC[3] = {1, 1, 1}, invC[3] = {1, 1, 1}, xFmin[3] = {0, 0, 0}, xCmin[3] = {0, 0, 0};
  if (cmask) {
#pragma unroll
    for (int d = 0; d < NDIM; ++d) {
      dxF[d] = A.dxb[3 * b + d];
      dxC[d] = 2.0 * dxF[d];
      invC[d] = 1.0 / dxC[d];
      xFmin[d] = A.bxmin[3 * b + d] - 2.0 * dxF[d];
      xCmin[d] = A.bxmin[3 * b + d] - 2.0 * dxC[d];
    }
  }
  const int total = s_off[nreg];
  for (int e = t; e < total; e += blockDim.x) {
    int lo = 0, hi = nreg - 1;  // region r with s_off[r] <= e < s_off[r+1]
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (s_off[mid] <= e) lo = mid;
      else hi = mid - 1;
    }
    const int q = s_q[lo], kind = s_kind[lo];
    const int dd[3] = {q % 3 - 1, (q / 3) % 3 - 1, q / 9 - 1};
    int li = e - s_off[lo];
    int gc[3] = {0, 0, 0};  // ghosted index 0..bn+3
#pragma unroll
    for (int d = 0; d < NDIM; ++d) {
      const int ext = dd[d] ? 2 : bn;
      const int l = li % ext;
      li /= ext;
      gc[d] = dd[d] < 0 ? l : (dd[d] > 0 ? bn + 2 + l : 2 + l);
    }
    double val[AMR_GHOST_VG];
    if (kind == AMR_COARSE) {  // prolongation (interpolation_linear)
      int pc[3] = {0, 0, 0};
      double eta[3] = {0, 0, 0};
#pragma unroll
      for (int d = 0; d < NDIM; ++d) {
        const double xF = xFmin[d] + (double(gc[d] + 1) - 0.5) * dxF[d];
        const int ixC = int((xF - xCmin[d]) * invC[d]) + 1;
        const double xC = xCmin[d] + (double(ixC) - 0.5) * dxC[d];
        eta[d] = (xF - xC) * invC[d];
        pc[d] = ixC - 1;
      }
#pragma unroll
      for (int vv = 0; vv < AMR_GHOST_VG; ++vv) {
        if (vv >= nv) break;
        const double *ps = psc + vv * CC;
        auto at = [&](int a, int bb, int cc) { return ps[a + C * (bb + CY * cc)]; };
        const double c0 = at(pc[0], pc[1], pc[2]);
        double x = c0;
        double slope[3] = {0, 0, 0};
#pragma unroll
        for (int d = 0; d < NDIM; ++d) {
          const int e0 = d == 0, e1 = d == 1, e2 = d == 2;
          const double sL = c0 - at(pc[0] - e0, pc[1] - e1, pc[2] - e2);
          const double sR = at(pc[0] + e0, pc[1] + e1, pc[2] + e2) - c0;
          const double sC = 0.5 * (sR + sL);
          const double sg = copysign(1.0, sC);
          slope[d] = sg * fmax(0.0, fmin(fmin(fabs(sC), sg * sL), sg * sR));
        }
#pragma unroll
        for (int d = 0; d < NDIM; ++d) x = x + slope[d] * eta[d];
        val[vv] = x;
      }
    } else {  // restriction
      int P[3] = {0, 0, 0};
#pragma unroll
      for (int d = 0; d < NDIM; ++d) P[d] = igb[d] * bn + gc[d] - 2;
      const CoarseSrc src = coarse_source<NDIM>(A, L, P[0], P[1], P[2]);
#pragma unroll
      for (int vv = 0; vv < AMR_GHOST_VG; ++vv)
        if (vv < nv) val[vv] = coarse_read<NDIM>(src, v0 + vv, bn);
    }
#pragma unroll
    for (int vv = 0; vv < AMR_GHOST_VG; ++vv)
      if (vv < nv) A.gbuf[ghost_offset<NDIM>(slot, A.nw, v0 + vv, gc[0] - 2, gc[1] - 2, gc[2] - 2, bn)] = val[vv];
  }
}

// fix_conserve (src/mod_fix_conserve.t:465-595): the boundary cells of a
// coarse block next to a finer one swap the coarse interface flux for the
// area average of the fine fluxes: w = w - pc, then w = w + pf / 2^d with pc
// and pf as store_flux keeps them; faces in the reference's order.
template <int NDIM>
__global__ void __launch_bounds__(256) amr_fix_kernel(const AmrFixArgs A) {
  const int slot = blockIdx.x;
  const int b = A.iblocks[slot];
  const int t = threadIdx.x;
  const double cofi = 1.0 / double(1 << NDIM);
  const int dsel = sweep_dir(A.sweep, A.split_xy, A.scal, NDIM);
  const int BN = A.bn;
  for (int d = 0; d < NDIM; ++d)
    for (int side = 0; side < 2; ++side) {
      if (dsel >= 0 && d != dsel) continue;
      int dd[3] = {0, 0, 0};
      dd[d] = side ? 1 : -1;
      const int q = dir_index(dd[0], dd[1], dd[2]);
      if (A.ntype[b * 27 + q] != AMR_FINE) continue;
      int ta = -1, tb = -1;
      for (int e = 0; e < NDIM; ++e)
        if (e != d) { if (ta < 0) ta = e; else tb = e; }
      const int n1 = BN, n2 = tb >= 0 ? BN : 1;
      const double *own = A.pflux + ((size_t)A.gslot[b] * (2 * NDIM) + 2 * d + side) * A.nw * (BN * BN);
      for (int p = t; p < A.nw * n1 * n2; p += blockDim.x) {
        const int v = p / (n1 * n2), a1 = p % n1, b2 = (p / n1) % n2;
        int c[3] = {0, 0, 0};
        c[d] = side ? BN - 1 : 0;
        c[ta] = a1;
        if (tb >= 0) c[tb] = b2;
        const double f = own[v * (BN * BN) + a1 + BN * b2];
        const double pc = side ? f : -f;
        int ic[3] = {0, 0, 0};
        ic[d] = side ? 0 : 1;
        ic[ta] = a1 >= BN / 2;
        if (tb >= 0) ic[tb] = b2 >= BN / 2;
        const int chd = A.child[(b * 27 + q) * 8 + ic[0] + 2 * ic[1] + 4 * ic[2]];
        const double *fp = A.pflux + ((size_t)A.gslot[chd] * (2 * NDIM) + 2 * d + (1 - side)) * A.nw * (BN * BN) +
                           v * (BN * BN);
        const int fa = 2 * (a1 - (BN / 2) * ic[ta]), fbb = tb >= 0 ? 2 * (b2 - (BN / 2) * ic[tb]) : 0;
        double sum = 0.0;
        bool first = true;
        for (int y = 0; y < (tb >= 0 ? 2 : 1); ++y)
          for (int x = 0; x < 2; ++x) {
            const double g = fp[fa + x + BN * (fbb + y)];
            sum = first ? g : sum + g;
            first = false;
          }
        const double pf = side ? sum : -sum;  // the fine block's side 1 - side
        double &w = A.w[cell_offset<NDIM>(b, A.nw, v, c[0], c[1], c[2], BN)];
        w = w - pc;
        w = w + pf * cofi;
      }
      __syncthreads();
    }
}

// Regrid (amr_coarsen_refine, src/amr/mod_coarsen_refine.t:20-182): one CTA
// per new leaf.  A refined child takes prolong_2nd (src/amr/mod_refine.t:
// 81-167): per coarse cell of its footprint in the parent, monotonized-central
// slopes from the parent's neighbours (across the parent's faces through the
// old tree's gather, i.e. its getbc ghost values), then
// w = wCo + (slope_1 eta_1) + (slope_2 eta_2) [+ (slope_3 eta_3)], left to
// right, eta = 0.5 (i - ixFi - 0.5) = -1/4 or +1/4.  A coarsened parent takes
// coarsen_grid of its children (src/amr/mod_coarsen.t:12-79): the average of
// 2^d fine cells, x fastest.
template <int NDIM>
__global__ void __launch_bounds__(256) amr_remap_kernel(const AmrRemapArgs A) {
  const StageArgs &S = A.old;
  const int BN = S.bn, half = BN / 2;
  const int NY = NDIM >= 2 ? BN : 1, NZ = NDIM >= 3 ? BN : 1, NC = BN * NY * NZ;
  const int nb = blockIdx.x;
  const int *op = A.op + 9 * nb;
  const int kind = op[0];
  for (int e = threadIdx.x; e < A.nw * NC; e += blockDim.x) {
    const int v = e / NC, cell = e - v * NC;
    const int i = cell % BN, j = NDIM >= 2 ? (cell / BN) % BN : 0, k = NDIM >= 3 ? cell / (BN * BN) : 0;
    double val;
    if (kind == 0) {
      val = S.uin[cell_offset<NDIM>(op[1], A.nw, v, i, j, k, BN)];
    } else if (kind == 1) {
      const int p = op[1], cb = op[2];
      const int co[3] = {(BN / 2) * (cb & 1) + (i >> 1), NDIM >= 2 ? (BN / 2) * ((cb >> 1) & 1) + (j >> 1) : 0,
                         NDIM >= 3 ? (BN / 2) * ((cb >> 2) & 1) + (k >> 1) : 0};
      auto wco = [&](int di, int dj, int dk) -> double {
        int ii = co[0] + di, jj = co[1] + dj, kk = co[2] + dk;
        uint32_t flip;
        const int blk = resolve_cell<NDIM>(S, p, ii, jj, kk, flip, BN);
        const double x = blk >= 0 ? S.uin[cell_offset<NDIM>(blk, A.nw, v, ii, jj, kk, BN)]
                                  : S.gbuf[ghost_offset<NDIM>(-2 - blk, A.nw, v, ii, jj, kk, BN)];
        return ((flip >> v) & 1u) ? -x : x;
      };
      const double c0 = wco(0, 0, 0);
      double slope[3] = {0, 0, 0};
#pragma unroll
      for (int d = 0; d < NDIM; ++d) {
        const int e0 = d == 0, e1 = d == 1, e2 = d == 2;
        const double sL = c0 - wco(-e0, -e1, -e2);
        const double sR = wco(e0, e1, e2) - c0;
        const double sC = 0.5 * (sR + sL);
        const double sg = copysign(1.0, sC);
        slope[d] = sg * fmax(0.0, fmin(fmin(fabs(sC), sg * sL), sg * sR));
      }
      const int f[3] = {i & 1, j & 1, k & 1};
      val = c0;
#pragma unroll
      for (int d = 0; d < NDIM; ++d) val = val + slope[d] * (0.5 * (double(f[d]) - 0.5));
    } else {
      const int ci = i >= half, cj = j >= half, ck = k >= half;
      const int cbit = ci | (NDIM >= 2 ? cj << 1 : 0) | (NDIM >= 3 ? ck << 2 : 0);
      const double *w = S.uin + cell_offset<NDIM>(op[1 + cbit], A.nw, v, 2 * (i - half * ci),
                                                  NDIM >= 2 ? 2 * (j - half * cj) : 0,
                                                  NDIM >= 3 ? 2 * (k - half * ck) : 0, BN);
      double sum = w[0];
      sum = sum + w[1];
      if constexpr (NDIM > 1) {
        sum = sum + w[BN];
        sum = sum + w[BN + 1];
      }
      if constexpr (NDIM > 2) {
        sum = sum + w[BN * BN];
        sum = sum + w[BN * BN + 1];
        sum = sum + w[BN * BN + BN];
        sum = sum + w[BN * BN + BN + 1];
      }
      val = sum * (1.0 / double(1 << NDIM));
    }
    A.unew[cell_offset<NDIM>(nb, A.nw, v, i, j, k, BN)] = val;
  }
}

cudaError_t launch_amr_remap(const AmrRemapArgs &A, int nnew, int ndim, cudaStream_t s) {
  if (nnew <= 0) return cudaSuccess;
  if (ndim == 2) amr_remap_kernel<2><<<nnew, 256, 0, s>>>(A);
  else amr_remap_kernel<3><<<nnew, 256, 0, s>>>(A);
  return cudaGetLastError();
}

cudaError_t prepare_amr_ghosts(int ndim, int bn) {
  const size_t c = (size_t)bn / 2 + 4;
  const int sm2 = (int)(sizeof(double) * AMR_GHOST_VG * c * c), sm3 = (int)(sm2 * c);
  const auto attr = cudaFuncAttributeMaxDynamicSharedMemorySize;
  if (bn == 16) {
    if (ndim == 2) return cudaFuncSetAttribute(amr_ghost_kernel<2, 16>, attr, sm2);
    return cudaFuncSetAttribute(amr_ghost_kernel<3, 16>, attr, sm3);
  }
  if (ndim == 2) return cudaFuncSetAttribute(amr_ghost_kernel<2>, attr, sm2);
  return cudaFuncSetAttribute(amr_ghost_kernel<3>, attr, sm3);
}

cudaError_t launch_amr_ghosts(const AmrGhostArgs &A, int nslots, int ndim, cudaStream_t s) {
  if (nslots <= 0) return cudaSuccess;
  const dim3 grid(nslots, (A.nw + AMR_GHOST_VG - 1) / AMR_GHOST_VG);
  const size_t c = (size_t)A.bn / 2 + 4;  // psc edge
  const size_t sm2 = sizeof(double) * AMR_GHOST_VG * c * c, sm3 = sm2 * c;
  if (A.bn == 16) {
    if (ndim == 2) amr_ghost_kernel<2, 16><<<grid, 256, sm2, s>>>(A);
    else amr_ghost_kernel<3, 16><<<grid, 256, sm3, s>>>(A);
  } else {
    if (ndim == 2) amr_ghost_kernel<2><<<grid, 256, sm2, s>>>(A);
    else amr_ghost_kernel<3><<<grid, 256, sm3, s>>>(A);
  }
  return cudaGetLastError();
}

cudaError_t launch_amr_fix(const AmrFixArgs &A, int nslots, int ndim, cudaStream_t s) {
  if (nslots <= 0) return cudaSuccess;
  if (ndim == 2) amr_fix_kernel<2><<<nslots, 256, 0, s>>>(A);
  else amr_fix_kernel<3><<<nslots, 256, 0, s>>>(A);
  return cudaGetLastError();
}

// Shared memory of lohner_staged_kernel: one ghosted block-variable (two
// layers) and the per-cell error sums.
static size_t lohner_smem(int ndim, int bn) {
  const size_t g = (size_t)bn + 4;
  const size_t ng = ndim == 3 ? g * g * g : g * g, nc = ndim == 3 ? (size_t)bn * bn * bn : (size_t)bn * bn;
  return sizeof(double) * (ng + nc);
}

cudaError_t launch_lohner(const LohnerArgs &A, int ndim, cudaStream_t s) {
  if (ndim != 2 && ndim != 3) return cudaErrorInvalidValue;
  const size_t sm = lohner_smem(ndim, A.sa.bn);
  if (sm <= 100 * 1024) {  // block edges up to 16 in 3-D, every edge in 2-D
    const auto attr = cudaFuncAttributeMaxDynamicSharedMemorySize;
    if (ndim == 2) {
      if (cudaError_t e = cudaFuncSetAttribute(lohner_staged_kernel<2>, attr, (int)sm)) return e;
      lohner_staged_kernel<2><<<A.sa.nblocks, 256, sm, s>>>(A);
    } else {
      if (cudaError_t e = cudaFuncSetAttribute(lohner_staged_kernel<3>, attr, (int)sm)) return e;
      lohner_staged_kernel<3><<<A.sa.nblocks, 256, sm, s>>>(A);
    }
    return cudaGetLastError();
  }
  if (ndim == 2) lohner_kernel<2><<<A.sa.nblocks, 256, 0, s>>>(A);
  else lohner_kernel<3><<<A.sa.nblocks, 256, 0, s>>>(A);
  return cudaGetLastError();
}

}  // namespace amrvac
