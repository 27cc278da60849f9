// DST kernels for transform length 192 (dst_kernels.cuh) and the one-launch
// level solve of a square 192-cell level (cluster_solve.cuh).
#include "cluster_solve.cuh"

namespace ibpm {
IBPM_DST_DEFINE(192)
IBPM_CLUSTER_DEFINE(192)
}  // namespace ibpm
