// small_values_method = 'average' (src/mod_small_values.t:89-144, dispatched
// by hd_handle_small_values, src/hd/mod_hd_phys.t:1476-1490, and
// mhd_handle_small_values_origin, src/mhd/mod_mhd_phys.t:2226-2241).
//
// The fix is not local: a flagged density or pressure becomes the mean of the
// unflagged values of the surrounding cube (half-width 1 ..
// small_values_daverage, clipped to the ghosted block), over
//   S1 the ghosted block's conserved cells when finite_volume converts them
//      to primitives (a flag anywhere also takes every cell's energy through
//      the pressure / internal-energy round trip),
//   S2 the reconstructed face-state arrays of each direction (their cube
//      reaches faces of other rows and planes, and the prefilled cell values
//      where no face was reconstructed, src/mod_finite_volume.t:176-186),
//   S3 the updated state on exit, whose cube reaches the output register's
//      ghost cells (what the time stepper's elementwise combinations left
//      there: a_base * base + b_in * in of the registers' ghost values),
//   S4 the same after the GLM source (add_source_glm ends with the fix),
//   S6 the primitives of getdt_courant (src/mod_dt.t:189-191).
// The fused stage kernel holds one plane of face states and no ghost cells
// of its output, so it only detects: sv_detect_kernel flags every block with
// a small value among its ghosted cells (S1, S6); the stage kernel flags
// blocks where S2-S4 fire; sv_stage_kernel then recomputes each flagged
// block's stage in the reference's whole-block order in global scratch and
// overwrites its output, and sv_getdt_kernel does getdt's part for the
// flagged blocks the getdt kernel skipped.  Runs with FP64, single-level
// grids, unsplit stages, the dwlimiter2 limiters, and GLM or no divB source.
#include "kernels.cuh"

namespace amrvac {

namespace {

// ghosted-block geometry of one block edge and dimension
struct SvGeo {
  int G, nd, cells;
  __device__ SvGeo(int bn, int nd_) : G(bn + 4), nd(nd_), cells(1) {
    for (int d = 0; d < nd; ++d) cells *= G;
  }
  __device__ void coords(int c, int *x) const {
    x[0] = c % G;
    x[1] = nd >= 2 ? (c / G) % G : 0;
    x[2] = nd >= 3 ? c / (G * G) : 0;
  }
  __device__ int id(int i, int j, int k) const { return i + G * (j + (nd >= 3 ? G * k : 0)); }
  __device__ int off(int d) const { return d == 0 ? 1 : (d == 1 ? G : G * G); }
};

// the conserved value of register reg at ghosted coordinates (gi, gj, gk) of
// block b, gathered as the stage kernel gathers (neighbours, physical sides)
template <int NW, int NDIM>
__device__ void sv_gather(const StageArgs &A, const double *reg, int b, int gi, int gj, int gk, double *w) {
  int i = gi - 2, j = NDIM >= 2 ? gj - 2 : 0, k = NDIM >= 3 ? gk - 2 : 0;
  uint32_t flip;
  const int blk = resolve_cell<NDIM>(A, b, i, j, k, flip, A.bn);
  for (int v = 0; v < NW; ++v) {
    const double x = blk >= 0 ? reg[cell_offset<NDIM>(blk, NW, v, i, j, k, A.bn)]
                              : A.gbuf[ghost_offset<NDIM>(-2 - blk, NW, v, i, j, k, A.bn)];
    w[v] = ((flip >> v) & 1u) ? -x : x;
  }
}

// phys_check_w on one cell of an array (component stride cs)
template <bool MHD, int NDIR, bool GLM>
__device__ void sv_check(const double *arr, size_t cs, int c, bool primitive, const PhysParams &P, bool &frho,
                         bool &fe) {
  using V = Vars<MHD, NDIR, GLM>;
  double w[V::NW];
  for (int v = 0; v < V::NW; ++v) w[v] = arr[v * cs + c];
  frho = w[V::RHO] < P.small_density;
  double m2 = w[V::M0] * w[V::M0];
  for (int q = 1; q < NDIR; ++q) m2 = m2 + w[V::M0 + q] * w[V::M0 + q];
  if (primitive) {
    fe = w[V::E] < P.small_pressure;
  } else if constexpr (MHD) {
    double b2 = w[V::B0] * w[V::B0];
    for (int q = 1; q < NDIR; ++q) b2 = b2 + w[V::B0 + q] * w[V::B0 + q];
    fe = w[V::E] - 0.5 * (m2 / w[V::RHO] + b2) < P.small_e;
  } else {
    fe = P.gamma_1 * (w[V::E] - 0.5 * m2 / w[V::RHO]) < P.small_pressure;
  }
}

// small_values_average of component iw (values x[c]) over the flagged cells:
// the smallest cube of half-width 1 .. dav holding an unflagged cell,
// clipped to the ghosted block, summed x fastest.  Flagged cells are only
// written and unflagged ones only read, so the threads need no order.
__device__ void sv_average(const SvGeo &g, double *x, const unsigned char *flag, int dav, double none_value,
                           bool has_none_value) {
  for (int c = threadIdx.x; c < g.cells; c += blockDim.x) {
    if (!flag[c]) continue;
    int ix[3];
    g.coords(c, ix);
    int lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    bool ok = false;
    for (int r = 1; r <= dav && !ok; ++r) {
      for (int d = 0; d < 3; ++d) {
        lo[d] = d < g.nd ? max(ix[d] - r, 0) : 0;
        hi[d] = d < g.nd ? min(ix[d] + r, g.G - 1) : 0;
      }
      for (int k = lo[2]; k <= hi[2] && !ok; ++k)
        for (int j = lo[1]; j <= hi[1] && !ok; ++j)
          for (int i = lo[0]; i <= hi[0] && !ok; ++i) ok = !flag[g.id(i, j, k)];
    }
    if (ok) {
      double sum = 0.0;
      int cnt = 0;
      for (int k = lo[2]; k <= hi[2]; ++k)
        for (int j = lo[1]; j <= hi[1]; ++j)
          for (int i = lo[0]; i <= hi[0]; ++i) {
            const int q = g.id(i, j, k);
            if (!flag[q]) {
              sum = sum + x[q];
              ++cnt;
            }
          }
      x[c] = sum / double(cnt);
    } else if (has_none_value) {
      x[c] = none_value;
    }
  }
}

// handle_small_values with method 'average' on a ghosted-block array arr
// (component stride g.cells) over the box [lo, hi] (ixO); the array is ixI.
// Returns true if any value was flagged.
template <bool MHD, int NDIR, bool GLM>
__device__ bool sv_handle(const SvGeo &g, double *arr, bool primitive, const int *lo, const int *hi,
                          unsigned char *frho, unsigned char *fe, const PhysParams &P, int *s_any) {
  using V = Vars<MHD, NDIR, GLM>;
  const size_t cs = g.cells;
  if (threadIdx.x == 0) *s_any = 0;
  __syncthreads();
  bool any = false;
  for (int c = threadIdx.x; c < g.cells; c += blockDim.x) {
    int x[3];
    g.coords(c, x);
    bool in = true;
    for (int d = 0; d < g.nd; ++d) in = in && x[d] >= lo[d] && x[d] <= hi[d];
    bool r = false, e = false;
    if (in) sv_check<MHD, NDIR, GLM>(arr, cs, c, primitive, P, r, e);
    frho[c] = r;
    fe[c] = e;
    any = any || r || e;
  }
  if (any) atomicOr(s_any, 1);
  __syncthreads();
  if (!*s_any) return false;
  const int dav = max(P.small_values_daverage, 1);
  sv_average(g, arr + V::RHO * cs, frho, dav, P.small_density, true);
  __syncthreads();
  auto m2_of = [&](int c) {
    double m2 = arr[V::M0 * cs + c] * arr[V::M0 * cs + c];
    for (int q = 1; q < NDIR; ++q) m2 = m2 + arr[(V::M0 + q) * cs + c] * arr[(V::M0 + q) * cs + c];
    return m2;
  };
  auto b2_of = [&](int c) {
    double b2 = 0.0;
    if constexpr (MHD) {
      b2 = arr[V::B0 * cs + c] * arr[V::B0 * cs + c];
      for (int q = 1; q < NDIR; ++q) b2 = b2 + arr[(V::B0 + q) * cs + c] * arr[(V::B0 + q) * cs + c];
    }
    return b2;
  };
  double *e = arr + V::E * cs;
  if (primitive) {
    sv_average(g, e, fe, dav, P.small_pressure, true);
    __syncthreads();
    return true;
  }
  // conserved: the energy as pressure (hd) or internal energy (mhd) over the
  // whole array, averaged, and back
  for (int c = threadIdx.x; c < g.cells; c += blockDim.x) {
    if constexpr (MHD) e[c] = e[c] - 0.5 * (m2_of(c) / arr[V::RHO * cs + c] + b2_of(c));
    else e[c] = P.gamma_1 * (e[c] - 0.5 * m2_of(c) / arr[V::RHO * cs + c]);
  }
  __syncthreads();
  sv_average(g, e, fe, dav, P.small_pressure, true);
  __syncthreads();
  for (int c = threadIdx.x; c < g.cells; c += blockDim.x) {
    if constexpr (MHD) e[c] = e[c] + 0.5 * (m2_of(c) / arr[V::RHO * cs + c] + b2_of(c));
    else e[c] = e[c] / P.gamma_1 + 0.5 * m2_of(c) / arr[V::RHO * cs + c];
  }
  __syncthreads();
  return true;
}

}  // namespace

// S1 / S6 detection: flags (ST_SV_AVG in block_status) every block with a
// small value among its ghosted conserved cells of register reg.
template <bool MHD, int NDIR, bool GLM, int NDIM>
__global__ void __launch_bounds__(256) sv_detect_kernel(const StageArgs A, const double *reg) {
  using V = Vars<MHD, NDIR, GLM>;
  const SvGeo g(A.bn, NDIM);
  for (int b = blockIdx.x; b < A.nblocks; b += gridDim.x) {
    bool any = false;
    for (int c = threadIdx.x; c < g.cells; c += blockDim.x) {
      int x[3];
      g.coords(c, x);
      double w[V::NW];
      sv_gather<V::NW, NDIM>(A, reg, b, x[0], x[1], x[2], w);
      bool r, e;
      sv_check<MHD, NDIR, GLM>(w, 1, 0, false, A.P, r, e);
      any = any || r || e;
    }
    if (__syncthreads_or(any) && threadIdx.x == 0) atomicOr(A.block_status + b, ST_SV_AVG);
  }
}

// Scratch of one CTA (SvScratch): the ghosted primitives, the two
// face-state arrays, the scaled face fluxes and the output state, each
// [NW][G^ndim], then two flag arrays of G^ndim bytes.

template <bool MHD, int NDIR, bool GLM, int NDIM, int SOLVER>
__global__ void __launch_bounds__(256) sv_stage_kernel(const StageArgs A, const double *snap_base,
                                                       const double *snap_in, SvScratch S) {
  using V = Vars<MHD, NDIR, GLM>;
  constexpr int NW = V::NW;
  const SvGeo g(A.bn, NDIM);
  const size_t cs = g.cells;
  double *Pa = S.base + (size_t)blockIdx.x * S.per_cta;
  double *L = Pa + NW * cs, *Rr = L + NW * cs, *FC = Rr + NW * cs, *WN = FC + NW * cs;
  unsigned char *f1 = reinterpret_cast<unsigned char *>(WN + NW * cs), *f2 = f1 + cs;
  __shared__ int s_any;
  const PhysParams &P = A.P;
  const double dt = *A.dt_dev, qdt = A.dtfactor * dt;
  const double cg = GLM ? *A.cmax_dev : 0.0;
  const double *rbase = snap_base ? snap_base : A.ubase;
  const double *rin = snap_in ? snap_in : A.uin;
  const int bn = A.bn;
  int ilo[3], ihi[3], all_lo[3] = {0, 0, 0}, all_hi[3] = {0, 0, 0};
  for (int d = 0; d < 3; ++d) {
    ilo[d] = d < NDIM ? 2 : 0;
    ihi[d] = d < NDIM ? bn + 1 : 0;
    all_hi[d] = d < NDIM ? bn + 3 : 0;
  }
  for (int b = blockIdx.x; b < A.nblocks; b += gridDim.x) {
    const uint32_t bs = A.block_status[b];
    if (!(bs & ST_SV_AVG)) {  // the stage kernel's result stands, and its status
      if ((bs & ST_NAN) && threadIdx.x == 0) atomicOr(A.status, ST_NAN);
      continue;
    }
    double dx[3], dxinv[3], rdel[3];
    for (int d = 0; d < 3; ++d) {
      dx[d] = d < NDIM ? A.dxb[b * 3 + d] : 1.0;
      dxinv[d] = -qdt / dx[d];
      const double r = P.cada3_radius * dx[d];
      const double a2m = P.schmid_global ? A.dt_dev[10 + d] : P.schmid_rad[d];
      rdel[d] = P.limiter == LIM_SCHMID ? (a2m + 1.0e-14) * (dx[d] * dx[d]) : 1.0 / (r * r);
    }
    // wCT and the RK combination a*base + b*in, ghost cells included
    for (int c = threadIdx.x; c < g.cells; c += blockDim.x) {
      int x[3];
      g.coords(c, x);
      double w[NW], wi[NW], wb[NW];
      sv_gather<NW, NDIM>(A, A.uin, b, x[0], x[1], x[2], w);
      sv_gather<NW, NDIM>(A, rin, b, x[0], x[1], x[2], wi);
      if (A.a_base != 0.0) sv_gather<NW, NDIM>(A, rbase, b, x[0], x[1], x[2], wb);
      for (int v = 0; v < NW; ++v) {
        Pa[v * cs + c] = w[v];
        WN[v * cs + c] = (A.a_base == 0.0) ? wi[v] : A.a_base * wb[v] + A.b_in * wi[v];
      }
    }
    __syncthreads();
    // S1: phys_to_primitive(ixI, ixI) with the small-value fix
    sv_handle<MHD, NDIR, GLM>(g, Pa, false, all_lo, all_hi, f1, f2, P, &s_any);
    for (int c = threadIdx.x; c < g.cells; c += blockDim.x) {
      double w[NW];
      for (int v = 0; v < NW; ++v) w[v] = Pa[v * cs + c];
      to_primitive<MHD, NDIR, GLM>(w, P);
      for (int v = 0; v < NW; ++v) Pa[v * cs + c] = w[v];
    }
    __syncthreads();
    for (int D = 0; D < NDIM; ++D) {
      const int o = g.off(D);
      // wLp = wprim, wRp = wprim shifted by one cell (the last layer unshifted)
      for (int c = threadIdx.x; c < g.cells; c += blockDim.x) {
        int x[3];
        g.coords(c, x);
        for (int v = 0; v < NW; ++v) {
          L[v * cs + c] = Pa[v * cs + c];
          Rr[v * cs + c] = x[D] < g.G - 1 ? Pa[v * cs + c + o] : Pa[v * cs + c];
        }
      }
      __syncthreads();
      // the faces ixCR: D from 1 to bn+1, transverse over the interior
      int flo[3], fhi[3];
      for (int d = 0; d < 3; ++d) {
        flo[d] = d == D ? 1 : ilo[d];
        fhi[d] = d == D ? bn + 1 : ihi[d];
      }
      for (int c = threadIdx.x; c < g.cells; c += blockDim.x) {
        int x[3];
        g.coords(c, x);
        bool in = true;
        for (int d = 0; d < NDIM; ++d) in = in && x[d] >= flo[d] && x[d] <= fhi[d];
        if (!in) continue;
        for (int v = 0; v < NW; ++v) {
          const double *q = Pa + v * cs;
          const double d0 = q[c] - q[c - o], d1 = q[c + o] - q[c], d2 = q[c + 2 * o] - q[c + o];
          double ldw, rdw;
          face_slopes<double, 0>(P.limiter, d0, d1, d2, rdel[D], ldw, rdw);
          L[v * cs + c] = q[c] + 0.5 * ldw;
          Rr[v * cs + c] = q[c + o] - 0.5 * rdw;
        }
      }
      __syncthreads();
      // S2: the reconstructed states (reconstruct_LR's handle_small_values)
      sv_handle<MHD, NDIR, GLM>(g, L, true, flo, fhi, f1, f2, P, &s_any);
      sv_handle<MHD, NDIR, GLM>(g, Rr, true, flo, fhi, f1, f2, P, &s_any);
      // fluxes of the faces, rotated as the stage kernel rotates them
      for (int c = threadIdx.x; c < g.cells; c += blockDim.x) {
        int x[3];
        g.coords(c, x);
        bool in = true;
        for (int d = 0; d < NDIM; ++d) in = in && x[d] >= flo[d] && x[d] <= fhi[d];
        if (!in) continue;
        double wl[NW], wr[NW], F[NW];
        for (int v = 0; v < NW; ++v) {
          const int ov = orig_index_rt<MHD, NDIR>(v, D);
          wl[v] = L[ov * cs + c];
          wr[v] = Rr[ov * cs + c];
        }
        face_from_states<double, MHD, NDIR, GLM, NDIM, SOLVER, 0>(wl, wr, P, cg, F, false);
        for (int v = 0; v < NW; ++v) FC[orig_index_rt<MHD, NDIR>(v, D) * cs + c] = dxinv[D] * F[v];
      }
      __syncthreads();
      // wnew += fC(i) - fC(i-1), in the stage kernel's order
      for (int c = threadIdx.x; c < g.cells; c += blockDim.x) {
        int x[3];
        g.coords(c, x);
        bool in = true;
        for (int d = 0; d < NDIM; ++d) in = in && x[d] >= ilo[d] && x[d] <= ihi[d];
        if (!in) continue;
        for (int v = 0; v < NW; ++v) WN[v * cs + c] = WN[v * cs + c] + FC[v * cs + c] - FC[v * cs + c - o];
      }
      __syncthreads();
    }
    // S3: the updated state, its cube reaching the output's ghost values
    sv_handle<MHD, NDIR, GLM>(g, WN, false, ilo, ihi, f1, f2, P, &s_any);
    if constexpr (MHD && GLM && NDIM > 1) {
      // add_source_glm (src/mhd/mod_mhd_phys.t:5472-5531), as the stage kernel
      const double qsrc = qdt;
      double mindx = dx[0];
      for (int d = 1; d < NDIM; ++d) mindx = fmin(mindx, dx[d]);
      for (int c = threadIdx.x; c < g.cells; c += blockDim.x) {
        int x[3];
        g.coords(c, x);
        bool in = true;
        for (int d = 0; d < NDIM; ++d) in = in && x[d] >= ilo[d] && x[d] <= ihi[d];
        if (!in) continue;
        double acc[NW];
        for (int v = 0; v < NW; ++v) acc[v] = WN[v * cs + c];
        if (P.glm_alpha < 0.0) {
          acc[V::PSI] = fabs(P.glm_alpha) * A.uin[cell_offset<NDIM>(b, NW, V::PSI, x[0] - 2, NDIM >= 2 ? x[1] - 2 : 0,
                                                                     NDIM >= 3 ? x[2] - 2 : 0, bn)];
        } else {
          acc[V::PSI] = exp(-(qsrc * cg * P.glm_alpha) / mindx) * acc[V::PSI];
        }
        if (P.glm_extended) {
          for (int d = 0; d < NDIM; ++d) {
            const int o = g.off(d);
            const double gq = ((Pa[V::PSI * cs + c + o] - Pa[V::PSI * cs + c - o]) * 0.5) / dx[d];
            acc[V::E] = acc[V::E] - qsrc * Pa[(V::B0 + d) * cs + c] * gq;
          }
          double divb = 0.0;
          for (int d = 0; d < NDIM; ++d) {
            const int o = g.off(d);
            divb = divb + 0.5 * (Pa[(V::B0 + d) * cs + c + o] - Pa[(V::B0 + d) * cs + c - o]) * (1.0 / dx[d]);
          }
          for (int q = 0; q < NDIR; ++q) acc[V::M0 + q] = acc[V::M0 + q] - qsrc * Pa[(V::B0 + q) * cs + c] * divb;
        }
        for (int v = 0; v < NW; ++v) WN[v * cs + c] = acc[v];
      }
      __syncthreads();
      // S4: add_source_glm's own fix
      sv_handle<MHD, NDIR, GLM>(g, WN, false, ilo, ihi, f1, f2, P, &s_any);
    }
    for (int c = threadIdx.x; c < g.cells; c += blockDim.x) {
      int x[3];
      g.coords(c, x);
      bool in = true;
      for (int d = 0; d < NDIM; ++d) in = in && x[d] >= ilo[d] && x[d] <= ihi[d];
      if (!in) continue;
      const int i = x[0] - 2, j = NDIM >= 2 ? x[1] - 2 : 0, k = NDIM >= 3 ? x[2] - 2 : 0;
      bool bad = false;
      for (int v = 0; v < NW; ++v) {
        const double y = WN[v * cs + c];
        A.uout[cell_offset<NDIM>(b, NW, v, i, j, k, bn)] = y;
        if ((v == V::RHO || v == V::E) && !isfinite(y)) bad = true;
      }
      if (bad) atomicOr(A.status, ST_NAN);
    }
    __syncthreads();
  }
}

// S6: getdt_courant of the flagged blocks (the getdt kernel skips them):
// the ghosted block through handle_small_values, then the interior's cmax
// reduced exactly as getdt_kernel reduces it.
template <bool MHD, int NDIR, bool GLM, int NDIM>
__global__ void __launch_bounds__(256) sv_getdt_kernel(const StageArgs A, const double *reg, int type_courant,
                                                        unsigned long long *red, SvScratch S) {
  using V = Vars<MHD, NDIR, GLM>;
  constexpr int NW = V::NW;
  const SvGeo g(A.bn, NDIM);
  const size_t cs = g.cells;
  double *Pa = S.base + (size_t)blockIdx.x * S.per_cta;
  unsigned char *f1 = reinterpret_cast<unsigned char *>(Pa + 5 * NW * cs), *f2 = f1 + cs;
  __shared__ int s_any;
  __shared__ double red_s[5][8];
  const int bn = A.bn;
  int all_lo[3] = {0, 0, 0}, all_hi[3] = {0, 0, 0};
  for (int d = 0; d < NDIM; ++d) all_hi[d] = bn + 3;
  for (int b = blockIdx.x; b < A.nblocks; b += gridDim.x) {
    if (!(A.block_status[b] & ST_SV_AVG)) continue;
    for (int c = threadIdx.x; c < g.cells; c += blockDim.x) {
      int x[3];
      g.coords(c, x);
      double w[NW];
      sv_gather<NW, NDIM>(A, reg, b, x[0], x[1], x[2], w);
      for (int v = 0; v < NW; ++v) Pa[v * cs + c] = w[v];
    }
    __syncthreads();
    sv_handle<MHD, NDIR, GLM>(g, Pa, false, all_lo, all_hi, f1, f2, A.P, &s_any);
    double dxinv[3];
    for (int d = 0; d < NDIM; ++d) dxinv[d] = 1.0 / A.dxb[b * 3 + d];
    double mtot = 0.0, mcm = 0.0, mdim[3] = {0.0, 0.0, 0.0};
    const int ncell = bn * (NDIM >= 2 ? bn : 1) * (NDIM == 3 ? bn : 1);
    for (int cc = threadIdx.x; cc < ncell; cc += blockDim.x) {
      const int i = cc % bn, j = NDIM >= 2 ? (cc / bn) % bn : 0, k = NDIM == 3 ? cc / (bn * bn) : 0;
      const int c = g.id(i + 2, NDIM >= 2 ? j + 2 : 0, NDIM >= 3 ? k + 2 : 0);
      double w[NW];
      for (int v = 0; v < NW; ++v) w[v] = Pa[v * cs + c];
      to_primitive<MHD, NDIR, GLM>(w, A.P);
      double tot = 0.0;
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
        const double cx = cm * dxinv[d];
        tot = d == 0 ? cx : tot + cx;
        mdim[d] = fmax(mdim[d], cx);
        mcm = fmax(mcm, cm);
      }
      mtot = fmax(mtot, tot);
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const double r0 = warp_max(mtot), r1 = warp_max(mcm);
    double r2[3];
    for (int d = 0; d < 3; ++d) r2[d] = warp_max(mdim[d]);
    if (lane == 0) {
      red_s[0][wid] = r0; red_s[1][wid] = r1;
      red_s[2][wid] = r2[0]; red_s[3][wid] = r2[1]; red_s[4][wid] = r2[2];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double a0 = 0, a1 = 0, d0 = 0, d1 = 0, d2 = 0;
      for (int q = 0; q < 8; ++q) {
        a0 = fmax(a0, red_s[0][q]); a1 = fmax(a1, red_s[1][q]);
        d0 = fmax(d0, red_s[2][q]); d1 = fmax(d1, red_s[3][q]); d2 = fmax(d2, red_s[4][q]);
      }
      double xr;
      if (type_courant == 1) {
        xr = a0;
      } else {
        const double dd[3] = {d0, d1, d2};
        double courantmax = 0.0, tot = 0.0;
        for (int d = 0; d < NDIM; ++d) {
          courantmax = fmax(courantmax, dd[d]);
          tot = tot + courantmax;
        }
        xr = type_courant == 2 ? tot : courantmax;
      }
      atomic_max_pos(red + 0, xr);
      atomic_max_pos(red + 1, a1);
    }
    __syncthreads();
  }
}

namespace {

template <bool MHD, int NDIR, bool GLM, int NDIM, int SOLVER>
struct SvLaunch {
  static cudaError_t detect(const StageArgs &A, const double *reg, cudaStream_t s) {
    sv_detect_kernel<MHD, NDIR, GLM, NDIM><<<A.nblocks < 1024 ? A.nblocks : 1024, 256, 0, s>>>(A, reg);
    return cudaGetLastError();
  }
  static cudaError_t stage(const StageArgs &A, const double *sb, const double *si, SvScratch S, int nctas,
                           cudaStream_t s) {
    sv_stage_kernel<MHD, NDIR, GLM, NDIM, SOLVER><<<nctas, 256, 0, s>>>(A, sb, si, S);
    return cudaGetLastError();
  }
  static cudaError_t getdt(const StageArgs &A, const double *reg, int tc, unsigned long long *red, SvScratch S,
                           int nctas, cudaStream_t s) {
    sv_getdt_kernel<MHD, NDIR, GLM, NDIM><<<nctas, 256, 0, s>>>(A, reg, tc, red, S);
    return cudaGetLastError();
  }
  static SvSet set() {
    SvSet k;
    k.detect = &detect;
    k.stage = &stage;
    k.getdt = &getdt;
    return k;
  }
};

template <bool MHD, int NDIR, bool GLM, int NDIM>
bool sv_solver(int solver, SvSet *out) {
  switch (solver) {
    case SOLVER_TVDLF: *out = SvLaunch<MHD, NDIR, GLM, NDIM, SOLVER_TVDLF>::set(); return true;
    case SOLVER_HLL: *out = SvLaunch<MHD, NDIR, GLM, NDIM, SOLVER_HLL>::set(); return true;
    case SOLVER_HLLC: *out = SvLaunch<MHD, NDIR, GLM, NDIM, SOLVER_HLLC>::set(); return true;
    case SOLVER_HLLD:
      if constexpr (MHD) { *out = SvLaunch<MHD, NDIR, GLM, NDIM, SOLVER_HLLD>::set(); return true; }
      return false;
    default: return false;
  }
}

}  // namespace

bool lookup_sv(const KernelKey &k, SvSet *out) {
  if (!k.mhd) {
    if (k.ndim == 2) return sv_solver<false, 2, false, 2>(k.solver, out);
    if (k.ndim == 3) return sv_solver<false, 3, false, 3>(k.solver, out);
    return false;
  }
  if (k.ndim == 2 && k.ndir == 2) return k.glm ? sv_solver<true, 2, true, 2>(k.solver, out)
                                               : sv_solver<true, 2, false, 2>(k.solver, out);
  if (k.ndim == 2 && k.ndir == 3) return k.glm ? sv_solver<true, 3, true, 2>(k.solver, out)
                                               : sv_solver<true, 3, false, 2>(k.solver, out);
  if (k.ndim == 3 && k.ndir == 3) return k.glm ? sv_solver<true, 3, true, 3>(k.solver, out)
                                               : sv_solver<true, 3, false, 3>(k.solver, out);
  return false;
}

}  // namespace amrvac
