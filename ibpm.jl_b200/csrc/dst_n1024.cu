// DST kernels for transform length 1024 (see dst_kernels.cuh).
#include "dst_kernels.cuh"

namespace ibpm {
IBPM_DST_DEFINE(1024)
}  // namespace ibpm
