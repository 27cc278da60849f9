// DST kernels for transform length 128 (see dst_kernels.cuh).
#include "dst_kernels.cuh"

namespace ibpm {
IBPM_DST_DEFINE(128)
}  // namespace ibpm
