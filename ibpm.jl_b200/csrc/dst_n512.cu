// DST kernels for transform length 512 (see dst_kernels.cuh).
#include "dst_kernels.cuh"

namespace ibpm {
IBPM_DST_DEFINE(512)
}  // namespace ibpm
