// Stage / getdt / point kernels for hydrodynamics (hd), 2-D and 3-D.
#include "kernels.cuh"

namespace amrvac {

bool lookup_hd(const KernelKey &k, KernelSet *out) {
  if (k.mhd || k.ndir != k.ndim) return false;
  if (k.mixed) {
    if (k.ndim == 2 && k.solver == SOLVER_HLLC && k.limiter == LIM_VANLEER && k.boundspeed == BS_EINFELDT) {
      *out = Launch<false, 2, false, 2, SOLVER_HLLC, LIM_VANLEER, BS_EINFELDT, float>::set();
      return true;
    }
    if (k.ndim == 2 && k.solver == SOLVER_HLLC) { *out = Launch<false, 2, false, 2, SOLVER_HLLC, 0, 0, float>::set(); return true; }
    if (k.ndim == 2 && k.solver == SOLVER_HLL) { *out = Launch<false, 2, false, 2, SOLVER_HLL, 0, 0, float>::set(); return true; }
    if (k.ndim == 3 && k.solver == SOLVER_HLLC) { *out = Launch<false, 3, false, 3, SOLVER_HLLC, 0, 0, float>::set(); return true; }
    return false;
  }
  // compile-time limiter / bound speed for the 2-D Kelvin-Helmholtz configuration
  if (k.ndim == 2 && k.solver == SOLVER_HLLC && k.limiter == LIM_VANLEER && k.boundspeed == BS_EINFELDT) {
    *out = Launch<false, 2, false, 2, SOLVER_HLLC, LIM_VANLEER, BS_EINFELDT>::set();
    return true;
  }
#define AMRVAC_HD(ND, S)                                        \
  if (k.ndim == ND && k.solver == S) {                          \
    *out = Launch<false, ND, false, ND, S>::set();              \
    return true;                                                \
  }
  AMRVAC_HD(2, SOLVER_TVDLF)
  AMRVAC_HD(2, SOLVER_TVDMU)
  AMRVAC_HD(3, SOLVER_TVDMU)
  AMRVAC_HD(2, SOLVER_HLL)
  AMRVAC_HD(2, SOLVER_HLLC)
  AMRVAC_HD(3, SOLVER_TVDLF)
  AMRVAC_HD(3, SOLVER_HLL)
  AMRVAC_HD(3, SOLVER_HLLC)
#undef AMRVAC_HD
  return false;
}

}  // namespace amrvac
