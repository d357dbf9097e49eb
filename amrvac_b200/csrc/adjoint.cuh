// Discrete adjoint of one explicit stage (declarations shared with capi.cu).
#pragma once

#include <cuda_runtime.h>

#include "stage.cuh"

namespace amrvac {

// One stage of the forward scheme is
//   W_new = a*B + b*W + sum_d s_d (F_{i-1/2} - F_{i+1/2}),  s_d = dtfactor*dt/dx_d,
// with F the fused face flux of W (reconstruction, Riemann solver).  Its
// adjoint for a frozen dt, given lam = dL/dW_new:
//   lam_out = acc_in + b*lam + (dF/dW)^T applied to the face weights
//             mu_f = s_d (lam_{right of f} - lam_{left of f}),
//   base    = (base_init ? 0 : base) + a*lam,
//   gamma_part[block] += dL/dgamma of this stage (per block, deterministic).
struct AdjArgs {
  StageArgs sa;            // sa.uin = W (stage input), nbr, bc, P
  const double *lam;       // dL/dW_new, register layout
  double *lam_out;         // dL/dW
  const double *acc_in;    // added into lam_out (may be null)
  double *base;            // base accumulator (may be null)
  int base_init;
  double a, b;
  double s[2];             // dtfactor*dt/dx per direction
  double *gamma_part;      // [nblocks]
};

// 2-D hydrodynamics, solver HLL (2) or HLLC (3), limiter minmod (1) or
// vanleer (5), Einfeldt bounds.
cudaError_t launch_adjoint_stage(const AdjArgs &A, int limiter, int solver, cudaStream_t s);
cudaError_t adjoint_prepare();
// *p = v on the stream (a device scalar without a host round trip)
cudaError_t launch_set_scalar(double *p, double v, cudaStream_t s);

}  // namespace amrvac
