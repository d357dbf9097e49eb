// Stage kernels with the fifth-order reconstructions (three-cell halo) for
// hydrodynamics, 2-D and 3-D, HLL and HLLC: MP5, and the WENO5 family (one
// kernel, variant at run time); and, on the two-cell halo, the WENO3 family
// and the Venkatakrishnan limiter.
#include "kernels.cuh"

namespace amrvac {

bool lookup_mp5_hd(const KernelKey &k, KernelSet *out) {
  if (k.mhd || k.mixed || k.ndir != k.ndim) return false;
#define AMRVAC_MP5_HD(ND, S)                                                              \
  if (k.ndim == ND && k.solver == S && k.limiter == LIM_MP5) {                            \
    *out = Launch<false, ND, false, ND, S, LIM_MP5>::set();                               \
    return true;                                                                          \
  }                                                                                       \
  if (k.ndim == ND && k.solver == S && k.limiter == LIM_WENO5) {                          \
    *out = Launch<false, ND, false, ND, S, LIM_WENO5>::set();                             \
    return true;                                                                          \
  }                                                                                       \
  if (k.ndim == ND && k.solver == S && k.limiter == LIM_WENO3) {                          \
    *out = Launch<false, ND, false, ND, S, LIM_WENO3>::set();                             \
    return true;                                                                          \
  }                                                                                       \
  if (k.ndim == ND && k.solver == S && k.limiter == LIM_VENK) {                           \
    *out = Launch<false, ND, false, ND, S, LIM_VENK>::set();                              \
    return true;                                                                          \
  }
  AMRVAC_MP5_HD(2, SOLVER_HLL)
  AMRVAC_MP5_HD(2, SOLVER_HLLC)
  AMRVAC_MP5_HD(3, SOLVER_HLL)
  AMRVAC_MP5_HD(3, SOLVER_HLLC)
#undef AMRVAC_MP5_HD
  return false;
}

}  // namespace amrvac
