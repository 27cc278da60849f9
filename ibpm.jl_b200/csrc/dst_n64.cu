// DST kernels for transform length 64 (dst_kernels.cuh) and the one-launch
// level solve of a square 64-cell level (cluster_solve.cuh).
#include "cluster_solve.cuh"

namespace ibpm {
IBPM_DST_DEFINE(64)
IBPM_CLUSTER_DEFINE(64)
}  // namespace ibpm
