// DST kernels for transform length 400 (see dst_kernels.cuh).
#include "dst_kernels.cuh"

namespace ibpm {
IBPM_DST_DEFINE(400)
}  // namespace ibpm
