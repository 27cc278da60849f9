// DST kernels for transform length 768 (see dst_kernels.cuh).
#include "dst_kernels.cuh"

namespace ibpm {
IBPM_DST_DEFINE(768)
}  // namespace ibpm
