// DST kernels for transform length 200 (see dst_kernels.cuh).
#include "dst_kernels.cuh"

namespace ibpm {
IBPM_DST_DEFINE(200)
}  // namespace ibpm
