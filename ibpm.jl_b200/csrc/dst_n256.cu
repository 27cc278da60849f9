// DST kernels for transform length 256 (dst_kernels.cuh) and the one-launch
// level solve of a square 256-cell level (cluster_solve.cuh).
#include "cluster_solve.cuh"

namespace ibpm {
IBPM_DST_DEFINE(256)
IBPM_CLUSTER_DEFINE(256)
}  // namespace ibpm
