// Kernels for block_nx = 8 (see k_blocks.cuh).
#include "k_blocks.cuh"

namespace amrvac {

bool lookup_bn8(const KernelKey &k, KernelSet *out) { return lookup_bn<8>(k, out); }

}  // namespace amrvac
