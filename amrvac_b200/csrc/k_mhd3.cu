// Stage / getdt / point kernels for ideal MHD in 3-D.
#include "kernels.cuh"

namespace amrvac {

bool lookup_mhd3(const KernelKey &k, KernelSet *out) {
  if (!k.mhd || k.ndim != 3 || k.ndir != 3) return false;
  if (k.mixed) {
    if (k.glm && k.solver == SOLVER_HLLD && k.limiter == LIM_CADA3 && k.boundspeed == BS_EINFELDT) {
      *out = Launch<true, 3, true, 3, SOLVER_HLLD, LIM_CADA3, BS_EINFELDT, float>::set();
      return true;
    }
    if (k.glm && k.solver == SOLVER_HLLD && k.limiter == LIM_VANLEER && k.boundspeed == BS_EINFELDT) {
      *out = Launch<true, 3, true, 3, SOLVER_HLLD, LIM_VANLEER, BS_EINFELDT, float>::set();
      return true;
    }
    if (k.glm && k.solver == SOLVER_HLLD) { *out = Launch<true, 3, true, 3, SOLVER_HLLD, 0, 0, float>::set(); return true; }
    if (k.glm && k.solver == SOLVER_HLL) { *out = Launch<true, 3, true, 3, SOLVER_HLL, 0, 0, float>::set(); return true; }
    return false;
  }
  // compile-time limiter / bound speed for the 3-D Orszag-Tang configuration
  // and the 3-D blast on the multi-level grid
  if (k.glm && k.solver == SOLVER_HLLD && k.limiter == LIM_CADA3 && k.boundspeed == BS_EINFELDT) {
    *out = Launch<true, 3, true, 3, SOLVER_HLLD, LIM_CADA3, BS_EINFELDT>::set();
    return true;
  }
  if (k.glm && k.solver == SOLVER_HLLD && k.limiter == LIM_VANLEER && k.boundspeed == BS_EINFELDT) {
    *out = Launch<true, 3, true, 3, SOLVER_HLLD, LIM_VANLEER, BS_EINFELDT>::set();
    return true;
  }
#define AMRVAC_M3(GLM, S)                                       \
  if (k.glm == GLM && k.solver == S) {                          \
    *out = Launch<true, 3, GLM, 3, S>::set();                   \
    return true;                                                \
  }
  AMRVAC_M3(false, SOLVER_TVDLF)
  AMRVAC_M3(false, SOLVER_HLL)
  AMRVAC_M3(false, SOLVER_HLLD)
  AMRVAC_M3(false, SOLVER_TVDMU)
  AMRVAC_M3(true, SOLVER_TVDLF)
  AMRVAC_M3(true, SOLVER_HLL)
  AMRVAC_M3(true, SOLVER_HLLD)
  AMRVAC_M3(false, SOLVER_HLLC)
  AMRVAC_M3(true, SOLVER_HLLC)
#undef AMRVAC_M3
  return false;
}

}  // namespace amrvac
