// DST kernels for transform length 512 (dst_kernels.cuh) and the one-launch
// level solve of a square 512-cell level (cluster_solve.cuh).
#include "cluster_solve.cuh"

namespace ibpm {
IBPM_DST_DEFINE(512)
IBPM_CLUSTER_DEFINE(512)
}  // namespace ibpm
