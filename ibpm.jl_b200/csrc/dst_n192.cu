// DST kernels for transform length 192 (see dst_kernels.cuh).
#include "dst_kernels.cuh"

namespace ibpm {
IBPM_DST_DEFINE(192)
}  // namespace ibpm
