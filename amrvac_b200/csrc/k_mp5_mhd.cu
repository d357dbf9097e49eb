// Stage kernels with the fifth-order reconstructions (three-cell halo) for
// MHD: 2-D with two or three vector components, 3-D; GLM or not; HLL and
// HLLD; MP5, the WENO5 and WENO3 families and the Venkatakrishnan limiter.
#include "kernels.cuh"

namespace amrvac {

bool lookup_mp5_mhd(const KernelKey &k, KernelSet *out) {
  if (!k.mhd || k.mixed) return false;
#define AMRVAC_MP5_M(ND, NDIR, GLM, S)                                                          \
  if (k.ndim == ND && k.ndir == NDIR && k.glm == GLM && k.solver == S && k.limiter == LIM_MP5) {  \
    *out = Launch<true, NDIR, GLM, ND, S, LIM_MP5>::set();                                      \
    return true;                                                                                \
  }                                                                                             \
  if (k.ndim == ND && k.ndir == NDIR && k.glm == GLM && k.solver == S && k.limiter == LIM_WENO5) { \
    *out = Launch<true, NDIR, GLM, ND, S, LIM_WENO5>::set();                                    \
    return true;                                                                                \
  }                                                                                             \
  if (k.ndim == ND && k.ndir == NDIR && k.glm == GLM && k.solver == S && k.limiter == LIM_WENO3) { \
    *out = Launch<true, NDIR, GLM, ND, S, LIM_WENO3>::set();                                    \
    return true;                                                                                \
  }                                                                                             \
  if (k.ndim == ND && k.ndir == NDIR && k.glm == GLM && k.solver == S && k.limiter == LIM_VENK) { \
    *out = Launch<true, NDIR, GLM, ND, S, LIM_VENK>::set();                                     \
    return true;                                                                                \
  }
  AMRVAC_MP5_M(2, 2, false, SOLVER_HLL)
  AMRVAC_MP5_M(2, 2, false, SOLVER_HLLD)
  AMRVAC_MP5_M(2, 3, true, SOLVER_HLL)
  AMRVAC_MP5_M(2, 3, true, SOLVER_HLLD)
  AMRVAC_MP5_M(3, 3, false, SOLVER_HLLD)
  AMRVAC_MP5_M(3, 3, true, SOLVER_HLL)
  AMRVAC_MP5_M(3, 3, true, SOLVER_HLLD)
#undef AMRVAC_MP5_M
  return false;
}

}  // namespace amrvac
