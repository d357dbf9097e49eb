// Declarations of the pool-transfer and setdt bookkeeping launchers.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "physics.cuh"

namespace amrvac {

// ixS_srl_/ixR_srl_ per dimension, 0-based in ghosted coordinates, indexed
// by direction+1 (src/mod_ghostcells_update.t:150-162).
struct SrlMaps {
  int smin[3][3], smax[3][3], rmin[3][3], rmax[3][3];
};
// Physical boundary per side: kind 0 periodic, 1 cont, 2 mirror; flip bitmask
// of variables that change sign (asymm).
struct BcSpec {
  int kind[6];
  uint32_t flip[6];
};

cudaError_t measure_fp64_peak(double *tflops);
cudaError_t run_wait_probe(int spins, uint32_t *flags);
// rcp_ / div_ / rcp_seed of the stage kernels on n device points (test entry).
cudaError_t launch_div_points(int n, const double *x, const double *y, double *q, double *r, double *seed,
                              cudaStream_t s);
cudaError_t launch_unpack(const double *src, double *pool, int first, int n, int nw, int ndim, int ng, int bn,
                          cudaStream_t s);
cudaError_t launch_pack(const double *pool, double *dst, int first, int n, int nw, int ndim, int ng, int bn,
                        const int *nbr, const SrlMaps &maps, const BcSpec &bc, const double *gbuf, cudaStream_t s);
cudaError_t launch_setdt_finalize(unsigned long long *red, double *scal, uint32_t *status, cudaStream_t s);
cudaError_t launch_advance_time(double *scal, cudaStream_t s);
cudaError_t launch_ssprk5_ps3(double *u3, const double *u2, const double *u1, double a53, double a54, size_t n,
                              cudaStream_t s);
cudaError_t launch_ssprk5_final(double *u0, const double *u1, const double *u2, const double *u3, double a55,
                                double r, double a41, double a44, size_t n, cudaStream_t s);
cudaError_t launch_rk4_combine(double *u0, const double *u1, const double *u2, const double *u3, size_t n,
                               cudaStream_t s);
cudaError_t launch_restore_blocks(const double *wct, double *wnew, const uint32_t *block_status, int nblocks,
                                  size_t per_block, cudaStream_t s);

}  // namespace amrvac
