// amrvac_gpu_getdt_noalloc: the CFL time-step reduction over blocks that the
// caller holds in its own device memory, using no device allocation at all.
//
// Who needs it: a host code whose device memory belongs to another runtime —
// e.g. an OpenACC or CUDA Fortran build of the AMR driver whose block arrays
// live in that runtime's pool, or a framework whose caching allocator reserves
// the device — may not call cudaMalloc/cudaFree itself, either because the
// memory is already claimed or because an allocation would synchronise the
// device in the middle of its time step.  Such a caller cannot create an
// amrvac_ctx (creation allocates the registers), but it can still ask for dt.
//
// Scratch: one file-scope device array (NOALLOC_SCRATCH_DOUBLES doubles,
// 1.25 MiB) that every GPU loading this library holds until exit.  It stages
// the per-block dx and holds one (courant, cmax) pair per block plus the final
// pair.  Every word a call reads is written earlier in the same call, so no
// part of it needs clearing.  All calls share it: calls that overlap on the
// GPU (two host threads, or two streams) race and may return each other's
// result.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <string>

#include "../../include/amrvac_gpu.h"
#include "kernels.cuh"

namespace amrvac {
int record_error(int code, const std::string &msg);  // capi.cu
}

using namespace amrvac;

namespace {

constexpr int MAXB = AMRVAC_NOALLOC_MAX_BLOCKS;
constexpr size_t OFF_DX = 0;                          // [MAXB][3] dx per block
constexpr size_t OFF_PART = 3 * (size_t)MAXB;         // [MAXB][2] per-block (courant, cmax)
constexpr size_t OFF_RES = 5 * (size_t)MAXB;          // [2] reduced (courant, cmax)
constexpr size_t NOALLOC_SCRATCH_DOUBLES = 5 * (size_t)MAXB + 32;

static __device__ __align__(256) double g_getdt_scratch[NOALLOC_SCRATCH_DOUBLES];

// The host-side name g_getdt_scratch is not a device address; the address is
// looked up once per device (with that device current) and cached here.
constexpr int MAX_DEVICES = 64;
double *g_scratch_dev[MAX_DEVICES] = {};
std::mutex g_scratch_mu;

int scratch_for_current_device(double **out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return record_error(AMRVAC_E_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= MAX_DEVICES) return record_error(AMRVAC_E_UNSUPPORTED, "device ordinal above 63");
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_dev[dev]) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_getdt_scratch);
    if (e != cudaSuccess)
      return record_error(AMRVAC_E_CUDA, std::string("cudaGetSymbolAddress(getdt scratch): ") + cudaGetErrorString(e));
    g_scratch_dev[dev] = static_cast<double *>(p);
  }
  *out = g_scratch_dev[dev];
  return 0;
}

// Per-block pass of getdt_courant (src/mod_dt.t:160-287): the same per-cell
// wave speeds and the same type_courant combination as getdt_kernel, but each
// block writes its (courant, cmax) pair to its own scratch slot instead of
// folding it into global atomics.
template <bool MHD, int NDIR, bool GLM, int NDIM>
__global__ void __launch_bounds__(256) getdt_blocks_kernel(const double *__restrict__ u, int bn, int type_courant,
                                                           PhysParams P, double *__restrict__ scratch) {
  using V = Vars<MHD, NDIR, GLM>;
  constexpr int NW = V::NW;
  const int ncell = bn * (NDIM >= 2 ? bn : 1) * (NDIM == 3 ? bn : 1);
  const int b = blockIdx.x;
  const int t = threadIdx.x;
  const double *dx = scratch + OFF_DX + (size_t)b * 3;
  double dxinv[3] = {0.0, 0.0, 0.0};
#pragma unroll
  for (int d = 0; d < NDIM; ++d) dxinv[d] = 1.0 / dx[d];
  // per thread: max of the cell sums, of cmax, and of cmax_d/dx_d per direction
  double msum = 0.0, mcm = 0.0, mdir[3] = {0.0, 0.0, 0.0};
  for (int c = t; c < ncell; c += 256) {  // the block's cells, x fastest
    const int i = c % bn, j = NDIM >= 2 ? (c / bn) % bn : 0, k = NDIM == 3 ? c / (bn * bn) : 0;
    double w[NW];
#pragma unroll
    for (int v = 0; v < NW; ++v) w[v] = __ldg(u + cell_offset<NDIM>(b, NW, v, i, j, k, bn));
    // phys_to_primitive with its small-value fix (src/mod_dt.t:189-191)
    if (P.fix_small_values) small_values<double, MHD, NDIR, GLM>(w, false, P);
    to_primitive<MHD, NDIR, GLM>(w, P);
    double sum = 0.0;
#pragma unroll
    for (int d = 0; d < NDIM; ++d) {
      double cm;
      if constexpr (MHD) {
        double cf;
        if (d == 0) cf = fast_speed<double, NDIR, V::B0 + 0>(w, P);
        else if (d == 1) cf = fast_speed<double, NDIR, V::B0 + (NDIR > 1 ? 1 : 0)>(w, P);
        else cf = fast_speed<double, NDIR, V::B0 + (NDIR > 2 ? 2 : 0)>(w, P);
        cm = fabs(w[V::M0 + d]) + cf;
      } else {
        cm = fabs(w[V::M0 + d]) + sqrt(P.gamma * w[V::E] / w[V::RHO]);
      }
      const double c = cm * dxinv[d];
      sum = d == 0 ? c : sum + c;
      mdir[d] = fmax(mdir[d], c);
      mcm = fmax(mcm, cm);
    }
    msum = fmax(msum, sum);
  }
  __shared__ double red[5][8];
  const int lane = t & 31, wid = t >> 5;
  const double r0 = warp_max(msum), r1 = warp_max(mcm);
  const double r2 = warp_max(mdir[0]), r3 = warp_max(mdir[1]), r4 = warp_max(mdir[2]);
  if (lane == 0) {
    red[0][wid] = r0; red[1][wid] = r1; red[2][wid] = r2; red[3][wid] = r3; red[4][wid] = r4;
  }
  __syncthreads();
  if (t == 0) {
    double a[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    for (int q = 0; q < 8; ++q)
      for (int r = 0; r < 5; ++r) a[r] = fmax(a[r], red[r][q]);
    double x;
    if (type_courant == 1) {  // maxsum
      x = a[0];
    } else {                  // summax (2) / minimum (3), running max over directions as the reference
      double courantmax = 0.0, tot = 0.0;
      for (int d = 0; d < NDIM; ++d) {
        courantmax = fmax(courantmax, a[2 + d]);
        tot = tot + courantmax;
      }
      x = type_courant == 2 ? tot : courantmax;
    }
    scratch[OFF_PART + 2 * (size_t)b + 0] = x;
    scratch[OFF_PART + 2 * (size_t)b + 1] = a[1];
  }
}

// Max of the per-block pairs over nblocks (one CTA), written to the result slot.
__global__ void __launch_bounds__(256) getdt_combine_kernel(int nblocks, double *__restrict__ scratch) {
  double x = 0.0, cm = 0.0;
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x) {
    x = fmax(x, scratch[OFF_PART + 2 * (size_t)b + 0]);
    cm = fmax(cm, scratch[OFF_PART + 2 * (size_t)b + 1]);
  }
  __shared__ double red[2][8];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  x = warp_max(x);
  cm = warp_max(cm);
  if (lane == 0) { red[0][wid] = x; red[1][wid] = cm; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a0 = 0.0, a1 = 0.0;
    for (int q = 0; q < 8; ++q) { a0 = fmax(a0, red[0][q]); a1 = fmax(a1, red[1][q]); }
    scratch[OFF_RES + 0] = a0;
    scratch[OFF_RES + 1] = a1;
  }
}

template <bool MHD, int NDIR, bool GLM, int NDIM>
cudaError_t launch_blocks(const double *u, int nblocks, int bn, int type_courant, const PhysParams &P,
                          double *scratch, cudaStream_t s) {
  getdt_blocks_kernel<MHD, NDIR, GLM, NDIM><<<nblocks, 256, 0, s>>>(u, bn, type_courant, P, scratch);
  return cudaGetLastError();
}

using BlocksFn = cudaError_t (*)(const double *, int, int, int, const PhysParams &, double *, cudaStream_t);

BlocksFn pick(const amrvac_cfg &k, bool glm) {
  if (k.physics == 0) {
    if (k.ndim == 2 && k.ndir == 2) return &launch_blocks<false, 2, false, 2>;
    if (k.ndim == 3 && k.ndir == 3) return &launch_blocks<false, 3, false, 3>;
    return nullptr;
  }
  if (k.ndim == 2 && k.ndir == 2) return glm ? &launch_blocks<true, 2, true, 2> : &launch_blocks<true, 2, false, 2>;
  if (k.ndim == 2 && k.ndir == 3) return glm ? &launch_blocks<true, 3, true, 2> : &launch_blocks<true, 3, false, 2>;
  if (k.ndim == 3 && k.ndir == 3) return glm ? &launch_blocks<true, 3, true, 3> : &launch_blocks<true, 3, false, 3>;
  return nullptr;
}

}  // namespace

extern "C" int amrvac_gpu_getdt_noalloc(const amrvac_cfg *cfg, const double *w_dev, int nblocks, const double *dx,
                                        void *stream, double *dt, double *cmax_global) {
  if (!cfg || !w_dev || !dx) return record_error(AMRVAC_E_ARG, "getdt_noalloc: null argument");
  if (nblocks <= 0) return record_error(AMRVAC_E_ARG, "getdt_noalloc: nblocks must be positive");
  if (nblocks > MAXB)
    return record_error(AMRVAC_E_ARG, "getdt_noalloc: nblocks " + std::to_string(nblocks) +
                                          " exceeds the scratch limit AMRVAC_NOALLOC_MAX_BLOCKS = " +
                                          std::to_string(MAXB));
  const amrvac_cfg &k = *cfg;
  if (k.physics != 0 && k.physics != 1) return record_error(AMRVAC_E_ARG, "getdt_noalloc: physics must be 0 or 1");
  if (k.type_courant < 1 || k.type_courant > 3) return record_error(AMRVAC_E_ARG, "getdt_noalloc: bad type_courant");
  const int bn = k.block_nx[0];
  for (int d = 0; d < k.ndim && d < 3; ++d)
    if (k.block_nx[d] != bn || bn < 4 || bn % 2 || bn > 1024)
      return record_error(AMRVAC_E_UNSUPPORTED,
                          "getdt_noalloc: block_nx must be even, >= 4 and the same in every direction");
  if (k.fix_small_values && k.small_values_method == 2)
    return record_error(AMRVAC_E_UNSUPPORTED,
                        "getdt_noalloc: small_values_method average needs the ghost cells of a context");
  const bool glm = k.physics == 1 && k.typedivbfix == AMRVAC_DIVB_GLM;
  BlocksFn fn = pick(k, glm);
  if (!fn) return record_error(AMRVAC_E_UNSUPPORTED, "getdt_noalloc: unsupported physics/ndim/ndir");
  PhysParams P{};
  P.gamma = k.gamma;
  P.gamma_1 = k.gamma - 1.0;
  P.inv_gamma_1 = 1.0 / (k.gamma - 1.0);
  P.courantpar = k.courantpar;

  double *scratch = nullptr;
  if (int r = scratch_for_current_device(&scratch)) return r;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  double res[2] = {0.0, 0.0};
  cudaError_t e = cudaMemcpyAsync(scratch + OFF_DX, dx, sizeof(double) * 3 * (size_t)nblocks,
                                  cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = fn(w_dev, nblocks, bn, k.type_courant, P, scratch, s);
  if (e == cudaSuccess) {
    getdt_combine_kernel<<<1, 256, 0, s>>>(nblocks, scratch);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(res, scratch + OFF_RES, sizeof(res), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return record_error(AMRVAC_E_CUDA, std::string("getdt_noalloc: ") + cudaGetErrorString(e));
  double d = 1.0e99;  // bigdouble; smalldouble 1e-12 as in setdt
  if (res[0] > 1.0e-12) d = std::min(d, k.courantpar / res[0]);
  if (dt) *dt = d;
  if (cmax_global) *cmax_global = res[1];
  return d < k.dtmin ? (int)AMRVAC_ST_DT_TOO_SMALL : 0;
}
