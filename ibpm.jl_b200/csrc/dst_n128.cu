// DST kernels for transform length 128 (dst_kernels.cuh) and the one-launch
// level solve of a square 128-cell level (cluster_solve.cuh).
#include "cluster_solve.cuh"

namespace ibpm {
IBPM_DST_DEFINE(128)
IBPM_CLUSTER_DEFINE(128)
}  // namespace ibpm
