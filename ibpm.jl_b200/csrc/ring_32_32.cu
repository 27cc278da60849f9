// Spectral level chain for 32 x 32 grids (see ring_kernels.cuh).
#include "ring_kernels.cuh"

namespace ibpm {
IBPM_RING_DEFINE(32, 32)
}  // namespace ibpm
