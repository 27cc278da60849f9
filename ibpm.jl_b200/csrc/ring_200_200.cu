// Spectral level chain for 200 x 200 grids (see ring_kernels.cuh).
#include "ring_kernels.cuh"

namespace ibpm {
IBPM_RING_DEFINE(200, 200)
}  // namespace ibpm
