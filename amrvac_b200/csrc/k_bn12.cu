// Kernels for block_nx = 12 (see k_blocks.cuh).
#include "k_blocks.cuh"

namespace amrvac {

bool lookup_bn12(const KernelKey &k, KernelSet *out) { return lookup_bn<12>(k, out); }

}  // namespace amrvac
