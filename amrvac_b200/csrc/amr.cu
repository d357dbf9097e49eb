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
  const int i = t & (BN - 1), j = NDIM >= 2 ? t >> 4 : 0;
  const StageArgs &S = A.sa;
  const int nw = A.nw;
  const int lev = A.level[b];
  const double wf = A.wavefilter[lev - 1], thr = A.threshold[lev - 1], der = A.derefine[lev - 1];
  auto wv = [&](int iw, int x, int y, int z) -> double {
    int ii = x, jj = y, kk = z;
    uint32_t flip;
    const int blk = resolve_cell<NDIM>(S, b, ii, jj, kk, flip);
    double v = S.uin[cell_offset<NDIM>(blk, nw, iw, ii, jj, kk)];
    if ((flip >> iw) & 1u) v = -v;
    return ((A.logflag >> iw) & 1u) ? log10(v) : v;
  };
  bool any_ref = false, all_coa = true;
  double emax = 0.0;
  const bool active = t < (NDIM >= 2 ? BN * BN : BN);
  const int nz = NDIM == 3 ? BN : 1;
  for (int k = 0; k < nz && active; ++k) {
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
  const int r_all = __syncthreads_and(active ? all_coa : true);
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
template <int NDIM>
__device__ double coarse_value(const AmrGhostArgs &A, int L, int P0, int P1, int P2, int v) {
  const int P[3] = {P0, P1, P2};
  int jg[3] = {0, 0, 0}, loc[3] = {0, 0, 0};
#pragma unroll
  for (int d = 0; d < NDIM; ++d) {
    const int n = A.nlev[L][d] * BN;
    const int p = ((P[d] % n) + n) % n;  // periodic domain
    jg[d] = p >> 4;
    loc[d] = p & (BN - 1);
  }
  const int o = A.owner[A.owner_off[L] + jg[0] + A.nlev[L][0] * (jg[1] + A.nlev[L][1] * jg[2])];
  if (o >= 0) return A.u[cell_offset<NDIM>(o, A.nw, v, loc[0], loc[1], loc[2])];
  if (o == -2 && L < A.maxlevel) {
    int jf[3] = {0, 0, 0}, f[3] = {0, 0, 0};
#pragma unroll
    for (int d = 0; d < NDIM; ++d) {
      const int c = loc[d] >> 3;
      jf[d] = 2 * jg[d] + c;
      f[d] = 2 * (loc[d] - 8 * c);
    }
    const int o2 = A.owner[A.owner_off[L + 1] + jf[0] + A.nlev[L + 1][0] * (jf[1] + A.nlev[L + 1][1] * jf[2])];
    if (o2 >= 0) {
      double sum = 0.0;
      bool first = true;
      for (int kk = 0; kk < (NDIM > 2 ? 2 : 1); ++kk)
        for (int jj = 0; jj < (NDIM > 1 ? 2 : 1); ++jj)
          for (int ii = 0; ii < 2; ++ii) {
            const double x = A.u[cell_offset<NDIM>(o2, A.nw, v, f[0] + ii, f[1] + jj, f[2] + kk)];
            sum = first ? x : sum + x;
            first = false;
          }
      return sum * (1.0 / double(1 << NDIM));
    }
  }
  atomicOr(A.status, ST_BOUNDS);  // hierarchy not 2:1 balanced here
  return 0.0;
}

template <int NDIM>
__global__ void __launch_bounds__(256) amr_ghost_kernel(const AmrGhostArgs A) {
  extern __shared__ double psc[];  // 12^NDIM coarse representation of one variable
  constexpr int G = BN + 4, GY = NDIM >= 2 ? G : 1, GZ = NDIM >= 3 ? G : 1;
  constexpr int C = BN / 2 + 4, CY = NDIM >= 2 ? C : 1, CZ = NDIM >= 3 ? C : 1;
  const int slot = blockIdx.x;
  const int b = A.iblocks[slot];
  const int t = threadIdx.x;
  const int L = A.level[b];
  const int *nt = A.ntype + b * 27;
  bool has_coarse = false;
  for (int q = 0; q < 27; ++q) has_coarse |= nt[q] == AMR_COARSE;
  int igb[3] = {0, 0, 0};
  double dxF[3] = {1, 1, 1}, dxC[3] = {1, 1, 1}, invC[3] = {1, 1, 1}, xFmin[3] = {0, 0, 0}, xCmin[3] = {0, 0, 0};
#pragma unroll
  for (int d = 0; d < NDIM; ++d) {
    igb[d] = A.ig[3 * b + d];
    dxF[d] = A.dxb[3 * b + d];
    dxC[d] = 2.0 * dxF[d];
    invC[d] = 1.0 / dxC[d];
    xFmin[d] = A.bxmin[3 * b + d] - 2.0 * dxF[d];
    xCmin[d] = A.bxmin[3 * b + d] - 2.0 * dxC[d];
  }
  for (int v = 0; v < A.nw; ++v) {
    if (has_coarse) {
      for (int p = t; p < C * CY * CZ; p += blockDim.x) {
        const int pc[3] = {p % C, (p / C) % CY, p / (C * CY)};
        // only the cells some prolongation stencil reads: the centre of a
        // ghost cell of a coarser-neighbour direction (coarse index 1 for
        // the low ghosts, 2..9 beside the block, 10 for the high ghosts) or
        // one of its axial neighbours
        bool needed = false;
        for (int m = 0; m <= 2 * NDIM && !needed; ++m) {
          int cc[3] = {pc[0], pc[1], pc[2]};
          if (m > 0) cc[(m - 1) >> 1] += (m & 1) ? 1 : -1;
          int dd[3] = {0, 0, 0};
          bool ok = true;
#pragma unroll
          for (int d = 0; d < NDIM; ++d) {
            if (cc[d] < 1 || cc[d] > BN / 2 + 2) ok = false;
            dd[d] = cc[d] == 1 ? -1 : (cc[d] == BN / 2 + 2 ? 1 : 0);
          }
          needed = ok && (dd[0] | dd[1] | dd[2]) && nt[dir_index(dd[0], dd[1], dd[2])] == AMR_COARSE;
        }
        if (!needed) continue;
        int P[3] = {0, 0, 0};
#pragma unroll
        for (int d = 0; d < NDIM; ++d) P[d] = igb[d] * (BN / 2) + pc[d] - 2;
        psc[p] = coarse_value<NDIM>(A, L - 1, P[0], P[1], P[2], v);
      }
    }
    __syncthreads();
    for (int g = t; g < G * GY * GZ; g += blockDim.x) {
      const int gc[3] = {g % G, (g / G) % GY, g / (G * GY)};
      int dir[3] = {0, 0, 0};
      bool inside = true;
#pragma unroll
      for (int d = 0; d < NDIM; ++d) {
        dir[d] = gc[d] < 2 ? -1 : (gc[d] >= BN + 2 ? 1 : 0);
        inside = inside && dir[d] == 0;
      }
      if (inside) continue;
      const int kind = nt[dir_index(dir[0], dir[1], dir[2])];
      double val;
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
        auto at = [&](int a, int bb, int cc) { return psc[a + C * (bb + CY * cc)]; };
        const double c0 = at(pc[0], pc[1], pc[2]);
        val = c0;
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
        for (int d = 0; d < NDIM; ++d) val = val + slope[d] * eta[d];
      } else if (kind == AMR_FINE) {  // restriction
        int P[3] = {0, 0, 0};
#pragma unroll
        for (int d = 0; d < NDIM; ++d) P[d] = igb[d] * BN + gc[d] - 2;
        val = coarse_value<NDIM>(A, L, P[0], P[1], P[2], v);
      } else {
        continue;
      }
      A.gbuf[ghost_offset<NDIM>(slot, A.nw, v, gc[0] - 2, gc[1] - 2, gc[2] - 2)] = val;
    }
    __syncthreads();
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
  for (int d = 0; d < NDIM; ++d)
    for (int side = 0; side < 2; ++side) {
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
        double &w = A.w[cell_offset<NDIM>(b, A.nw, v, c[0], c[1], c[2])];
        w = w - pc;
        w = w + pf * cofi;
      }
      __syncthreads();
    }
}

cudaError_t launch_amr_ghosts(const AmrGhostArgs &A, int nslots, int ndim, cudaStream_t s) {
  if (nslots <= 0) return cudaSuccess;
  if (ndim == 2) amr_ghost_kernel<2><<<nslots, 256, sizeof(double) * 12 * 12, s>>>(A);
  else amr_ghost_kernel<3><<<nslots, 256, sizeof(double) * 12 * 12 * 12, s>>>(A);
  return cudaGetLastError();
}

cudaError_t launch_amr_fix(const AmrFixArgs &A, int nslots, int ndim, cudaStream_t s) {
  if (nslots <= 0) return cudaSuccess;
  if (ndim == 2) amr_fix_kernel<2><<<nslots, 256, 0, s>>>(A);
  else amr_fix_kernel<3><<<nslots, 256, 0, s>>>(A);
  return cudaGetLastError();
}

cudaError_t launch_lohner(const LohnerArgs &A, int ndim, cudaStream_t s) {
  if (ndim == 2) lohner_kernel<2><<<A.sa.nblocks, 256, 0, s>>>(A);
  else if (ndim == 3) lohner_kernel<3><<<A.sa.nblocks, 256, 0, s>>>(A);
  else return cudaErrorInvalidValue;
  return cudaGetLastError();
}

}  // namespace amrvac
