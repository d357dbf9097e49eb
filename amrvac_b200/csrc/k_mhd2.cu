// Stage / getdt / point kernels for ideal MHD in 2-D (ndir 2 or 3, i.e. 2.5D).
#include "kernels.cuh"

namespace amrvac {

bool lookup_mhd2(const KernelKey &k, KernelSet *out) {
  if (!k.mhd || k.ndim != 2) return false;
  if (k.mixed) {
    if (k.ndir == 3 && k.glm && k.solver == SOLVER_HLLD && k.limiter == LIM_CADA3 && k.boundspeed == BS_EINFELDT) {
      *out = Launch<true, 3, true, 2, SOLVER_HLLD, LIM_CADA3, BS_EINFELDT, float>::set();
      return true;
    }
    if (k.ndir == 3 && k.glm && k.solver == SOLVER_HLLD) { *out = Launch<true, 3, true, 2, SOLVER_HLLD, 0, 0, float>::set(); return true; }
    if (k.ndir == 3 && !k.glm && k.solver == SOLVER_HLL) { *out = Launch<true, 3, false, 2, SOLVER_HLL, 0, 0, float>::set(); return true; }
    return false;
  }
  // compile-time limiter / bound speed for the field-loop regression schemes
  if (k.ndir == 3 && k.glm && k.solver == SOLVER_HLLD && k.limiter == LIM_CADA3 && k.boundspeed == BS_EINFELDT) {
    *out = Launch<true, 3, true, 2, SOLVER_HLLD, LIM_CADA3, BS_EINFELDT>::set();
    return true;
  }
#define AMRVAC_M2(NDIR, GLM, S)                                 \
  if (k.ndir == NDIR && k.glm == GLM && k.solver == S) {        \
    *out = Launch<true, NDIR, GLM, 2, S>::set();                \
    return true;                                                \
  }
  AMRVAC_M2(2, false, SOLVER_TVDLF)
  AMRVAC_M2(2, false, SOLVER_HLL)
  AMRVAC_M2(2, false, SOLVER_HLLD)
  AMRVAC_M2(2, false, SOLVER_TVDMU)
  AMRVAC_M2(3, false, SOLVER_TVDMU)
  AMRVAC_M2(2, true, SOLVER_TVDLF)
  AMRVAC_M2(2, true, SOLVER_HLL)
  AMRVAC_M2(2, true, SOLVER_HLLD)
  AMRVAC_M2(3, false, SOLVER_TVDLF)
  AMRVAC_M2(3, false, SOLVER_HLL)
  AMRVAC_M2(3, false, SOLVER_HLLD)
  AMRVAC_M2(3, true, SOLVER_TVDLF)
  AMRVAC_M2(3, true, SOLVER_HLL)
  AMRVAC_M2(3, true, SOLVER_HLLD)
  AMRVAC_M2(2, false, SOLVER_HLLC)
  AMRVAC_M2(2, true, SOLVER_HLLC)
  AMRVAC_M2(3, false, SOLVER_HLLC)
  AMRVAC_M2(3, true, SOLVER_HLLC)
#undef AMRVAC_M2
  return false;
}

}  // namespace amrvac
