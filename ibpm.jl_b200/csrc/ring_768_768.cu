// Spectral level chain for 768 x 768 grids (see ring_kernels.cuh).
#include "ring_kernels.cuh"

namespace ibpm {
IBPM_RING_DEFINE(768, 768)
}  // namespace ibpm
