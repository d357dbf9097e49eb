// Kernels for block_nx = 10 (see k_blocks.cuh).
#include "k_blocks.cuh"

namespace amrvac {

bool lookup_bn10(const KernelKey &k, KernelSet *out) { return lookup_bn<10>(k, out); }

}  // namespace amrvac
