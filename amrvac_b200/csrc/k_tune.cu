// Stage-kernel variants of the benchmark schemes, timed by the autotuner
// (amrvac_gpu_autotune) next to the default kernel of the scheme's set:
// 3-D MHD HLLD + Einfeldt + GLM with cada3 (Orszag-Tang) or vanleer (the
// multi-level blast) at block_nx 16, FP64 and mixed.
//   FP64:  1 = 256 threads x 2 CTAs/SM, asynchronous plane staging
//          2 = 288 threads x 2 CTAs/SM (one round per x and y face phase)
//          3 = 256 threads x 1 CTA/SM (no register cap)
//   mixed: 1 = 256 x 2, 2 = 256 x 4, 3 = 288 x 3
#include "kernels.cuh"

namespace amrvac {

template <class TF, int LIM>
static void add_mhd3(KernelSet *out) {
  StageVar<true, 3, true, 3, SOLVER_HLLD, LIM, BS_EINFELDT, TF, BN16, 1>::add(*out, 1);
  StageVar<true, 3, true, 3, SOLVER_HLLD, LIM, BS_EINFELDT, TF, BN16, 2>::add(*out, 2);
  StageVar<true, 3, true, 3, SOLVER_HLLD, LIM, BS_EINFELDT, TF, BN16, 3>::add(*out, 3);
}

bool add_stage_variants(const KernelKey &k, KernelSet *out) {
  if (!(k.mhd && k.ndim == 3 && k.ndir == 3 && k.glm && k.solver == SOLVER_HLLD && k.boundspeed == BS_EINFELDT &&
        k.bn == BN16))
    return false;
  if (k.limiter == LIM_CADA3) {
    if (k.mixed) add_mhd3<float, LIM_CADA3>(out);
    else add_mhd3<double, LIM_CADA3>(out);
    return true;
  }
  if (k.limiter == LIM_VANLEER) {
    if (k.mixed) add_mhd3<float, LIM_VANLEER>(out);
    else add_mhd3<double, LIM_VANLEER>(out);
    return true;
  }
  return false;
}

}  // namespace amrvac
