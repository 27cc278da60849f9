// Spectral level chain for 128 x 64 grids (see ring_kernels.cuh).
#include "ring_kernels.cuh"

namespace ibpm {
IBPM_RING_DEFINE(128, 64)
}  // namespace ibpm
