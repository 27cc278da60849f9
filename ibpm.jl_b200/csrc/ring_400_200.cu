// Spectral level chain for 400 x 200 grids (see ring_kernels.cuh).
#include "ring_kernels.cuh"

namespace ibpm {
IBPM_RING_DEFINE(400, 200)
}  // namespace ibpm
