// DST kernels for transform length 32 (see dst_kernels.cuh).
#include "dst_kernels.cuh"

namespace ibpm {
IBPM_DST_DEFINE(32)
}  // namespace ibpm
