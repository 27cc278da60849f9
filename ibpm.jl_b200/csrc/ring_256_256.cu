// Spectral level chain for 256 x 256 grids (see ring_kernels.cuh).
#include "ring_kernels.cuh"

namespace ibpm {
IBPM_RING_DEFINE(256, 256)
}  // namespace ibpm
