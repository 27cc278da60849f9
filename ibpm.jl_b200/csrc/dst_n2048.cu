// DST kernels for transform length 2048 (see dst_kernels.cuh).
#include "dst_kernels.cuh"

namespace ibpm {
IBPM_DST_DEFINE(2048)
}  // namespace ibpm
