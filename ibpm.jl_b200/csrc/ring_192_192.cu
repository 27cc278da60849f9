// Spectral level chain for 192 x 192 grids (see ring_kernels.cuh).
#include "ring_kernels.cuh"

namespace ibpm {
IBPM_RING_DEFINE(192, 192)
}  // namespace ibpm
