// Stage / getdt / point kernels for hydrodynamics (hd), 2-D and 3-D.
#include "kernels.cuh"

namespace amrvac {

bool lookup_hd(const KernelKey &k, KernelSet *out) {
  if (k.mhd || k.ndir != k.ndim) return false;
#define AMRVAC_HD(ND, S)                                        \
  if (k.ndim == ND && k.solver == S) {                          \
    *out = Launch<false, ND, false, ND, S>::set();              \
    return true;                                                \
  }
  AMRVAC_HD(2, SOLVER_TVDLF)
  AMRVAC_HD(2, SOLVER_HLL)
  AMRVAC_HD(2, SOLVER_HLLC)
  AMRVAC_HD(3, SOLVER_TVDLF)
  AMRVAC_HD(3, SOLVER_HLL)
  AMRVAC_HD(3, SOLVER_HLLC)
#undef AMRVAC_HD
  return false;
}

}  // namespace amrvac
