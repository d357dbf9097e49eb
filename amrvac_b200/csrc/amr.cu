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

cudaError_t launch_lohner(const LohnerArgs &A, int ndim, cudaStream_t s) {
  if (ndim == 2) lohner_kernel<2><<<A.sa.nblocks, 256, 0, s>>>(A);
  else if (ndim == 3) lohner_kernel<3><<<A.sa.nblocks, 256, 0, s>>>(A);
  else return cudaErrorInvalidValue;
  return cudaGetLastError();
}

}  // namespace amrvac
