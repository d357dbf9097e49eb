// AMR decision kernels (declarations shared with capi.cu).
#pragma once

#include <cuda_runtime.h>

#include "stage.cuh"

namespace amrvac {

constexpr int AMR_MAX_LEVELS = 20;

struct LohnerArgs {
  StageArgs sa;                         // sa.uin = the register, nbr, bc
  int nw;
  double weight[16];                    // w_refine_weight per conserved variable
  uint32_t logflag;                     // bit iw: use log10 of variable iw
  double wavefilter[AMR_MAX_LEVELS];    // amr_wavefilter per level
  double threshold[AMR_MAX_LEVELS];     // refine_threshold per level
  double derefine[AMR_MAX_LEVELS];      // derefine_ratio per level
  const int *level;                     // [nblocks] 1-based level
  int refine_max_level;
  int *flags;                           // [nblocks] 1 refine | 2 coarsen
  double *errmax;                       // [nblocks] largest error of the block
};

cudaError_t launch_lohner(const LohnerArgs &A, int ndim, cudaStream_t s);

}  // namespace amrvac
