// Spectral level chain for 128 x 128 grids (see ring_kernels.cuh).
#include "ring_kernels.cuh"

namespace ibpm {
IBPM_RING_DEFINE(128, 128)
}  // namespace ibpm
