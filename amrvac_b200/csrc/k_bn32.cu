// Kernels for block_nx = 32 (see k_blocks.cuh).
#include "k_blocks.cuh"

namespace amrvac {

bool lookup_bn32(const KernelKey &k, KernelSet *out) { return lookup_bn<32>(k, out); }

}  // namespace amrvac
