// Spectral level chain for 384 x 384 grids (see ring_kernels.cuh).
#include "ring_kernels.cuh"

namespace ibpm {
IBPM_RING_DEFINE(384, 384)
}  // namespace ibpm
