// Stage kernels with MP5 reconstruction (three-cell halo) for hydrodynamics,
// 2-D and 3-D, HLL and HLLC.
#include "kernels.cuh"

namespace amrvac {

bool lookup_mp5_hd(const KernelKey &k, KernelSet *out) {
  if (k.mhd || k.mixed || k.limiter != LIM_MP5 || k.ndir != k.ndim) return false;
#define AMRVAC_MP5_HD(ND, S)                                          \
  if (k.ndim == ND && k.solver == S) {                                \
    *out = Launch<false, ND, false, ND, S, LIM_MP5>::set();           \
    return true;                                                      \
  }
  AMRVAC_MP5_HD(2, SOLVER_HLL)
  AMRVAC_MP5_HD(2, SOLVER_HLLC)
  AMRVAC_MP5_HD(3, SOLVER_HLL)
  AMRVAC_MP5_HD(3, SOLVER_HLLC)
#undef AMRVAC_MP5_HD
  return false;
}

}  // namespace amrvac
