// DST kernels for transform length 384 (dst_kernels.cuh) and the one-launch
// level solve of a square 384-cell level (cluster_solve.cuh).
#include "cluster_solve.cuh"

namespace ibpm {
IBPM_DST_DEFINE(384)
IBPM_CLUSTER_DEFINE(384)
}  // namespace ibpm
