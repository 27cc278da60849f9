// DST kernels for transform length 400 (dst_kernels.cuh) and the one-launch
// level solve of a square 400-cell level (cluster_solve.cuh).
#include "cluster_solve.cuh"

namespace ibpm {
IBPM_DST_DEFINE(400)
IBPM_CLUSTER_DEFINE(400)
}  // namespace ibpm
