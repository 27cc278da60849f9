// Spectral level chain for 1024 x 1024 grids (see ring_kernels.cuh).
#include "ring_kernels.cuh"

namespace ibpm {
IBPM_RING_DEFINE(1024, 1024)
}  // namespace ibpm
