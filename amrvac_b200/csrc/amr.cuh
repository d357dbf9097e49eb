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

// Static multi-level grid (level jumps between leaf blocks, 2:1 balanced,
// periodic domain).  Neighbour kinds per block and direction.
enum : int { AMR_BOUNDARY = 0, AMR_COARSE = 1, AMR_SIBLING = 2, AMR_FINE = 3 };

struct AmrGhostArgs {
  const double *u;          // the register whose ghosts are needed
  double *gbuf;             // [slot][var][gz][gy][gx]
  int nw;
  const int *iblocks;       // [nslots] block of each slot
  const int *ntype;         // [nblocks*27]
  const int *level;         // [nblocks] 1-based
  const int *ig;            // [nblocks*3] block index at its level
  const double *bxmin;      // [nblocks*3] lower corner
  const double *dxb;        // [nblocks*3] cell size
  const int *owner;         // per level: leaf id, -2 refined, -1 covered by a coarser leaf
  int owner_off[AMR_MAX_LEVELS + 2];
  int nlev[AMR_MAX_LEVELS + 2][3];  // blocks per direction per level
  int maxlevel;
  int bn;                   // block edge
  int bc_kind[6];           // BCK_* per side (periodic sides wrap)
  uint32_t bc_flip[6];      // per side, bit v: variable v changes sign (asymm)
  uint32_t *status;
};

struct AmrFixArgs {
  double *w;                // the stage's output register
  const double *pflux;      // [slot][2*ndim][var][bn*bn]
  int nw;
  int bn;                   // block edge
  const int *iblocks, *gslot, *ntype, *child;  // child[(b*27+q)*8 + cbits]
  // dimensional splitting: only the sweep's direction (fix_conserve with
  // idim^LIM = idim, idim); sweep < 0: all directions
  int sweep, split_xy;
  const double *scal;
};

// Regrid: the state of the new tree's leaves from the old tree's register 0.
// op[9*b]: 0 copy of old leaf op[1]; 1 child op[2] (bits x, y, z) of old
// leaf op[1], by prolong_2nd; 2 parent of the old leaves op[1..2^d] (child
// bits order), by coarsen_grid.
struct AmrRemapArgs {
  StageArgs old;        // the old tree: uin = old register 0, nbr, gbuf (ghost pass done)
  const int *op;        // [nnew][9]
  double *unew;         // the new register 0
  int nw;
};

// Variables per CTA of the level-jump ghost pass.
constexpr int AMR_GHOST_VG = 3;
cudaError_t launch_amr_ghosts(const AmrGhostArgs &A, int nslots, int ndim, cudaStream_t s);
// Opt the ghost-pass kernel of (ndim, block edge) into its shared memory
// (AMR_GHOST_VG coarse representations); once per grid set-up.
cudaError_t prepare_amr_ghosts(int ndim, int bn);
// (the remap and Löhner kernels read the block edge from their StageArgs)
cudaError_t launch_amr_remap(const AmrRemapArgs &A, int nnew, int ndim, cudaStream_t s);
cudaError_t launch_amr_fix(const AmrFixArgs &A, int nslots, int ndim, cudaStream_t s);

}  // namespace amrvac
