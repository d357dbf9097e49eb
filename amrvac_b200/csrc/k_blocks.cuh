// Stage / getdt / point kernels for block edges other than 16 (block_nx 8,
// 10, 12, 32: the reference's own 3-D blast and Kelvin-Helmholtz and 2-D
// Riemann tests run 8^3, 10^3 and 12^2 blocks).  The slope limiters and
// bound speeds at run time (LIM = 0, BS = 0); FP64 with every solver
// (TVD-MUSCL with its MUSCL-Hancock predictor), the mixed form with the
// schemes it has at block edge 16.  Each block edge is instantiated in its
// own translation unit (k_bn*.cu) so that they compile in parallel.
#pragma once

#include "kernels.cuh"

namespace amrvac {

template <int BN>
bool lookup_bn(const KernelKey &k, KernelSet *out) {
  if (k.bn != BN) return false;
  if (k.mixed) {
    if (!k.mhd) {
      if (k.ndir != k.ndim) return false;
      if (k.ndim == 2 && k.solver == SOLVER_HLLC) { *out = Launch<false, 2, false, 2, SOLVER_HLLC, 0, 0, float, BN>::set(); return true; }
      if (k.ndim == 2 && k.solver == SOLVER_HLL) { *out = Launch<false, 2, false, 2, SOLVER_HLL, 0, 0, float, BN>::set(); return true; }
      if (k.ndim == 3 && k.solver == SOLVER_HLLC) { *out = Launch<false, 3, false, 3, SOLVER_HLLC, 0, 0, float, BN>::set(); return true; }
      return false;
    }
    if (k.ndim == 2 && k.ndir == 3 && k.glm && k.solver == SOLVER_HLLD) {
      *out = Launch<true, 3, true, 2, SOLVER_HLLD, 0, 0, float, BN>::set();
      return true;
    }
    if (k.ndim == 2 && k.ndir == 3 && !k.glm && k.solver == SOLVER_HLL) {
      *out = Launch<true, 3, false, 2, SOLVER_HLL, 0, 0, float, BN>::set();
      return true;
    }
    if (k.ndim == 3 && k.ndir == 3 && k.glm && k.solver == SOLVER_HLLD) {
      *out = Launch<true, 3, true, 3, SOLVER_HLLD, 0, 0, float, BN>::set();
      return true;
    }
    if (k.ndim == 3 && k.ndir == 3 && k.glm && k.solver == SOLVER_HLL) {
      *out = Launch<true, 3, true, 3, SOLVER_HLL, 0, 0, float, BN>::set();
      return true;
    }
    return false;
  }
  if (!k.mhd) {
    if (k.ndir != k.ndim) return false;
#define AMRVAC_BHD(ND, S)                                              \
    if (k.ndim == ND && k.solver == S) {                                 \
      *out = Launch<false, ND, false, ND, S, 0, 0, double, BN>::set();   \
      return true;                                                       \
    }
    AMRVAC_BHD(2, SOLVER_TVDLF)
    AMRVAC_BHD(2, SOLVER_HLL)
    AMRVAC_BHD(2, SOLVER_HLLC)
    AMRVAC_BHD(2, SOLVER_TVDMU)
    AMRVAC_BHD(3, SOLVER_TVDLF)
    AMRVAC_BHD(3, SOLVER_HLL)
    AMRVAC_BHD(3, SOLVER_HLLC)
    AMRVAC_BHD(3, SOLVER_TVDMU)
#undef AMRVAC_BHD
    return false;
  }
#define AMRVAC_BM(ND, NDIR, GLM, S)                                      \
  if (k.ndim == ND && k.ndir == NDIR && k.glm == GLM && k.solver == S) { \
    *out = Launch<true, NDIR, GLM, ND, S, 0, 0, double, BN>::set();       \
    return true;                                                          \
  }
#define AMRVAC_BM4(ND, NDIR, GLM)            \
  AMRVAC_BM(ND, NDIR, GLM, SOLVER_TVDLF)     \
  AMRVAC_BM(ND, NDIR, GLM, SOLVER_HLL)       \
  AMRVAC_BM(ND, NDIR, GLM, SOLVER_HLLC)      \
  AMRVAC_BM(ND, NDIR, GLM, SOLVER_HLLD)
  AMRVAC_BM4(2, 2, false)
  AMRVAC_BM4(2, 2, true)
  AMRVAC_BM4(2, 3, false)
  AMRVAC_BM4(2, 3, true)
  AMRVAC_BM4(3, 3, false)
  AMRVAC_BM4(3, 3, true)
  // TVD-MUSCL without GLM, as at block edge 16
  AMRVAC_BM(2, 2, false, SOLVER_TVDMU)
  AMRVAC_BM(2, 3, false, SOLVER_TVDMU)
  AMRVAC_BM(3, 3, false, SOLVER_TVDMU)
#undef AMRVAC_BM4
#undef AMRVAC_BM
  return false;
}

}  // namespace amrvac
