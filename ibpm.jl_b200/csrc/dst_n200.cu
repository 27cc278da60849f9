// DST kernels for transform length 200 (dst_kernels.cuh) and the one-launch
// level solve of a square 200-cell level (cluster_solve.cuh).
#include "cluster_solve.cuh"

namespace ibpm {
IBPM_DST_DEFINE(200)
IBPM_CLUSTER_DEFINE(200)
}  // namespace ibpm
