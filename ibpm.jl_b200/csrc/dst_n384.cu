// DST kernels for transform length 384 (see dst_kernels.cuh).
#include "dst_kernels.cuh"

namespace ibpm {
IBPM_DST_DEFINE(384)
}  // namespace ibpm
