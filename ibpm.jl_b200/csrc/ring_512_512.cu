// Spectral level chain for 512 x 512 grids (see ring_kernels.cuh).
#include "ring_kernels.cuh"

namespace ibpm {
IBPM_RING_DEFINE(512, 512)
}  // namespace ibpm
