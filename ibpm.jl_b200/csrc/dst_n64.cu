// DST kernels for transform length 64 (see dst_kernels.cuh).
#include "dst_kernels.cuh"

namespace ibpm {
IBPM_DST_DEFINE(64)
}  // namespace ibpm
