// DST kernels for transform length 256 (see dst_kernels.cuh).
#include "dst_kernels.cuh"

namespace ibpm {
IBPM_DST_DEFINE(256)
}  // namespace ibpm
