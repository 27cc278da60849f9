// One FP32 Poisson-type solve x = S((S r) ./ M .* scale) of a whole square
// level in ONE launch: a cluster of 16 CTAs holds the level in distributed
// shared memory (an FP32 level of 511² is 1 MB; 16 × 227 KB is 3.6 MB).
//
//   phase 1  CTA k transforms its rows [R k, R k + R) along x (DST-I, two
//            rows per group as in dst_x_kernel) and pushes each row's
//            column block d to the tile of CTA d (float4 stores to the
//            peer's shared memory);
//   phase 2  CTA k holds columns [R k, R k + R) of every row in its tile:
//            DST-I along y, spectral divide, DST-I along y (dst_y_kernel's
//            arithmetic on the tile);
//   phase 3  CTA k pulls its rows back from the 16 tiles, transforms them
//            along x and stores them (the correction of one refinement
//            sweep: ψ += d, or P += d and Γ −= P).
//
// Cluster barriers separate the phases; the last one keeps every CTA's
// shared memory alive until its peers have read it.  The right-hand side is
// the FP32 residual of the refinement (made by resid_kernel); on the vort2flux
// level chain the change of the coarser level's ψ enters through the edge
// terms apply_bc!(get_bc!(d_coarse)) (mg-utils.jl:7-60), d_coarse the FP32
// correction that the coarser level's solve stored.
#pragma once

#include <cooperative_groups.h>

#include "dst_kernels.cuh"

namespace ibpm {
namespace dstk {

constexpr int CS_CLUSTER = 16;
constexpr int CS_TP = 32;   // one warp per line pair: group barriers are __syncwarp, so 16 groups fit one CTA

template <int N>
__host__ __device__ constexpr int cs_rows() {   // rows (and columns) per CTA, even
    return ((((N - 1) + CS_CLUSTER - 1) / CS_CLUSTER) + 1) / 2 * 2;
}
template <int N>
__host__ __device__ constexpr int cs_groups() { return cs_rows<N>() / 2; }
template <int N>
__host__ __device__ constexpr int cs_threads() { return cs_groups<N>() * CS_TP; }
template <int N>
__host__ __device__ constexpr int cs_pitch() {  // tile pitch (floats): 16-byte rows, not a multiple of 32
    return ((cs_rows<N>() + 3) / 4) * 4 + 4 + ((((cs_rows<N>() + 3) / 4) * 4 + 4) % 32 == 0 ? 4 : 0);
}
template <int N>
__host__ __device__ constexpr bool cs_supported() { return cs_threads<N>() <= 1024; }

// Shared memory: tables | ay (n2) | tile (n2 × pitch) | FFT buffers | row staging
template <int N>
__host__ __device__ constexpr size_t cs_off_ay() { return tables_bytes<N, float>(); }
template <int N>
__host__ __device__ constexpr size_t cs_off_tile() {   // 16-byte aligned: the tile moves as float4
    return ((cs_off_ay<N>() + (size_t)round4(N) * 4 + 15) / 16) * 16;
}
template <int N>
__host__ __device__ constexpr size_t cs_off_buf() {
    return ((cs_off_tile<N>() + (size_t)(N - 1) * cs_pitch<N>() * 4 + 15) / 16) * 16;
}
template <int N>
__host__ __device__ constexpr size_t cs_off_stage() {
    return cs_off_buf<N>() + (size_t)cs_groups<N>() * ct_buf(N) * sizeof(float2);
}
template <int N>
__host__ __device__ constexpr size_t cs_smem() { return cs_off_stage<N>() + (size_t)cs_groups<N>() * 2 * N * 4; }

// get_bc! of an FP32 coarse field (the coarser level's correction).
__device__ __forceinline__ float getbc32_x(const float* rc, int P, int v, int c0, int jfix) {
    if ((v & 1) == 0) return rc[(long long)jfix * P + c0 + (v >> 1)];
    const int ia = c0 + ((v + 1) >> 1);
    return 0.5f * (rc[(long long)jfix * P + ia] + rc[(long long)jfix * P + ia - 1]);
}
__device__ __forceinline__ float getbc32_y(const float* rc, int P, int v, int c0, int ifix) {
    if ((v & 1) == 0) return rc[(long long)(c0 + (v >> 1)) * P + ifix];
    const int ja = c0 + ((v + 1) >> 1);
    return 0.5f * (rc[(long long)ja * P + ifix] + rc[(long long)(ja - 1) * P + ifix]);
}

template <int N, int EMIT>
__global__ void __launch_bounds__(cs_threads<N>(), 1) cluster_solve_kernel(ClusterSolveArgs a, Geom g, DstPlan p) {
    namespace cg = cooperative_groups;
    using V = float2;
    constexpr int TP = CS_TP;
    constexpr int R = cs_rows<N>();
    constexpr int G = cs_groups<N>();
    constexpr int TPITCH = cs_pitch<N>();
    constexpr int NQ = R / 4 + (R % 4 ? 1 : 0);   // float4 chunks per row block
    cg::cluster_group cl = cg::this_cluster();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V* tw = reinterpret_cast<V*>(smem_raw);
    float* sn = reinterpret_cast<float*>(tw + ct_tw_count(N));
    float* ay = reinterpret_cast<float*>(smem_raw + cs_off_ay<N>());
    float* tile = reinterpret_cast<float*>(smem_raw + cs_off_tile<N>());
    V* bufs = reinterpret_cast<V*>(smem_raw + cs_off_buf<N>());
    float* stage = reinterpret_cast<float*>(smem_raw + cs_off_stage<N>());
    const int n1 = g.n1, n2 = g.n2, P = g.P;
    const int rank = (int)cl.block_rank();
    const int y = blockIdx.y;                    // slab (one cluster per slab)
    const int lev = a.rmap.level(y);
    const Tabs<float> tb = tabs_of<float>(p);
    stage_tables<N, float>(tw, sn, tb);
    for (int j = threadIdx.x; j < n2; j += blockDim.x) cp_async4(ay + j, tb.c + j);
    cp_async_wait();
    __syncthreads();
    cl.sync();                                   // every CTA of the cluster runs before peers touch its tile
    pdl_wait();
    pdl_trigger();
    const int gid = threadIdx.x / TP, tid = threadIdx.x % TP;
    V* buf = bufs + gid * ct_buf(N);
    const int la = rank * R + 2 * gid;           // this group's rows la, la+1
    const bool va = la < n2, vb = la + 1 < n2;

    // ---- phase 1: rows along x, pushed to the owners of their column blocks
    if (va) {
        const float* r0 = a.r + a.rmap.off(y) + (long long)la * P;
        const float* dc = a.dc ? a.dc + a.dcmap.off(y) : nullptr;
        auto edge = [&](int i, int j) -> float {   // apply_bc!(get_bc!(d_coarse)) at (i, j)
            float v = 0.0f;
            if (j == 0) v += getbc32_x(dc, P, i + 1, g.nx / 4 - 1, g.ny / 4 - 1);
            if (j == n2 - 1) v += getbc32_x(dc, P, i + 1, g.nx / 4 - 1, 3 * g.ny / 4 - 1);
            if (i == 0) v += getbc32_y(dc, P, j + 1, g.ny / 4 - 1, g.nx / 4 - 1);
            if (i == n1 - 1) v += getbc32_y(dc, P, j + 1, g.ny / 4 - 1, 3 * g.nx / 4 - 1);
            return v;
        };
        auto load = [&](int i) -> V {
            float u = r0[i], w = vb ? r0[i + P] : 0.0f;
            if (dc) {
                if (la == 0 || la == n2 - 1 || i == 0 || i == n1 - 1) u += edge(i, la);
                if (vb && (la + 1 == n2 - 1 || i == 0 || i == n1 - 1)) w += edge(i, la + 1);
            }
            return V{u, w};
        };
        dst_pair<N, TP, cs_groups<N>(), float>(buf, tw, sn, tid, gid, load, [&](int o, V v) { buf[ct_pad(o)] = v; });
        gsync<TP, cs_groups<N>()>(gid);
        for (int idx = tid; idx < 2 * CS_CLUSTER * NQ; idx += TP) {
            const int pr = idx / (CS_CLUSTER * NQ), rem = idx % (CS_CLUSTER * NQ);
            const int d = rem / NQ, q = rem % NQ;
            if (pr == 1 && !vb) continue;
            float v4[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int c = d * R + 4 * q + u;
                const V z = (4 * q + u < R && c < n1) ? buf[ct_pad(c)] : V{0.0f, 0.0f};
                v4[u] = pr ? z.y : z.x;
            }
            float* peer = cl.map_shared_rank(tile, d);
            *reinterpret_cast<float4*>(peer + (long long)(la + pr) * TPITCH + 4 * q) =
                make_float4(v4[0], v4[1], v4[2], v4[3]);
        }
    }
    cl.sync();

    // ---- phase 2: columns [R rank, R rank + R) along y, divide, along y
    {
        const int ca = 2 * gid;                  // local column pair
        const int ia = rank * R + ca;            // global column
        if (ia < n1) {
            const bool hasb = ia + 1 < n1;
            auto load = [&](int m) -> V { return V{tile[m * TPITCH + ca], tile[m * TPITCH + ca + 1]}; };
            auto emit = [&](int o, V v) {
                tile[o * TPITCH + ca] = v.x;
                tile[o * TPITCH + ca + 1] = v.y;
            };
            dst_pair<N, TP, cs_groups<N>(), float>(buf, tw, sn, tid, gid, load, emit);
            gsync<TP, cs_groups<N>()>(gid);
            const float axa = __ldg(&tb.c[ia]);
            const float axb = hasb ? __ldg(&tb.c[ia + 1]) : 0.0f;
            const float kf = (a.sp.mode == SPEC_DELTA) ? 0.0f : (float)(a.sp.dt / a.sp.den[lev]);
            const float sc = (float)a.sp.scale;
            for (int o = tid; o < n2; o += TP) {
                const float l0 = axa + ay[o], l1 = axb + ay[o];
                const float M0 = (a.sp.mode == SPEC_DELTA) ? l0 : fmaf(l0, kf, 1.0f);
                const float M1 = (a.sp.mode == SPEC_DELTA) ? l1 : fmaf(l1, kf, 1.0f);
                tile[o * TPITCH + ca] *= __frcp_rn(M0) * sc;
                tile[o * TPITCH + ca + 1] = hasb ? tile[o * TPITCH + ca + 1] * (__frcp_rn(M1) * sc) : 0.0f;
            }
            gsync<TP, cs_groups<N>()>(gid);
            dst_pair<N, TP, cs_groups<N>(), float>(buf, tw, sn, tid, gid, load, emit);
        }
    }
    cl.sync();

    // ---- phase 3: rows back along x; the correction is added in FP64
    if (va) {
        float* st = stage + (size_t)gid * 2 * N;
        for (int idx = tid; idx < 2 * CS_CLUSTER * NQ; idx += TP) {
            const int pr = idx / (CS_CLUSTER * NQ), rem = idx % (CS_CLUSTER * NQ);
            const int d = rem / NQ, q = rem % NQ;
            if (pr == 1 && !vb) continue;
            if (4 * q >= R) continue;
            const float* peer = cl.map_shared_rank(tile, d);
            const float4 v = *reinterpret_cast<const float4*>(peer + (long long)(la + pr) * TPITCH + 4 * q);
            float* row = st + pr * N + d * R + 4 * q;
            const int c0 = d * R + 4 * q;
            if (c0 + 0 < N && 4 * q + 0 < R) row[0] = v.x;
            if (c0 + 1 < N && 4 * q + 1 < R) row[1] = v.y;
            if (c0 + 2 < N && 4 * q + 2 < R) row[2] = v.z;
            if (c0 + 3 < N && 4 * q + 3 < R) row[3] = v.w;
        }
        gsync<TP, cs_groups<N>()>(gid);
        constexpr int EO = (N - 1 + TP - 1) / TP;
        const long long ooff = a.out_map.off(y) + (long long)la * P;
        double* oa = a.out + ooff;
        double* xa = (EMIT == XEMIT_ACC_SUB) ? a.aux + a.aux_map.off(y) + (long long)la * P : nullptr;
        double po[EO][2];                        // the values the store updates, fetched under the FFT
#pragma unroll
        for (int k = 0; k < EO; ++k) {
            const int o = tid + k * TP;
            if (o < n1) {
                po[k][0] = oa[o];
                po[k][1] = vb ? oa[o + P] : 0.0;
            }
        }
        auto load = [&](int i) -> V { return V{st[i], vb ? st[N + i] : 0.0f}; };
        dst_pair<N, TP, cs_groups<N>(), float>(buf, tw, sn, tid, gid, load, [&](int o, V v) { buf[ct_pad(o)] = v; });
        gsync<TP, cs_groups<N>()>(gid);
        float* ds = a.dstore ? a.dstore + a.dstore_map.off(y) + (long long)la * P : nullptr;
#pragma unroll
        for (int k = 0; k < EO; ++k) {
            const int o = tid + k * TP;
            if (o >= n1) break;
            const V v = buf[ct_pad(o)];
            if constexpr (EMIT == XEMIT_ADD) {
                oa[o] = po[k][0] + (double)v.x;
                if (vb) oa[o + P] = po[k][1] + (double)v.y;
                if (ds) {
                    ds[o] = v.x;
                    if (vb) ds[o + P] = v.y;
                }
            } else {  // XEMIT_ACC_SUB
                const double pa = xa[o] + (double)v.x;
                xa[o] = pa;
                oa[o] = po[k][0] - pa;
                if (vb) {
                    const double pb = xa[o + P] + (double)v.y;
                    xa[o + P] = pb;
                    oa[o + P] = po[k][1] - pb;
                }
            }
        }
    }
    cl.sync();                                   // peers may still read this CTA's tile
}

template <int N>
cudaError_t cluster_attr_t() {
    if constexpr (!cs_supported<N>()) {
        return cudaErrorNotSupported;
    } else {
        cudaError_t e;
        for (auto k : {cluster_solve_kernel<N, XEMIT_ADD>, cluster_solve_kernel<N, XEMIT_ACC_SUB>}) {
            if ((e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cs_smem<N>())))
                return e;
            if ((e = cudaFuncSetAttribute(k, cudaFuncAttributeNonPortableClusterSizeAllowed, 1))) return e;
        }
        // can the device place one cluster of this kernel at all?
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(CS_CLUSTER, 1);
        cfg.blockDim = dim3(cs_threads<N>());
        cfg.dynamicSmemBytes = cs_smem<N>();
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = CS_CLUSTER;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        int nc = 0;
        if ((e = cudaOccupancyMaxActiveClusters(&nc, cluster_solve_kernel<N, XEMIT_ADD>, &cfg))) return e;
        return nc >= 1 ? cudaSuccess : cudaErrorNotSupported;
    }
}

template <int N>
cudaError_t cluster_launch_t(const Geom& g, const DstPlan& p, const ClusterSolveArgs& a, int nslabs,
                             cudaStream_t st) {
    if constexpr (!cs_supported<N>()) {
        return cudaErrorNotSupported;
    } else {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(CS_CLUSTER, nslabs);
        cfg.blockDim = dim3(cs_threads<N>());
        cfg.dynamicSmemBytes = cs_smem<N>();
        cfg.stream = st;
        cudaLaunchAttribute at[2];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = CS_CLUSTER;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        at[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        at[1].val.programmaticStreamSerializationAllowed = pdl_enabled() ? 1 : 0;
        cfg.attrs = at;
        cfg.numAttrs = 2;
        if (a.emit == XEMIT_ACC_SUB) return cudaLaunchKernelEx(&cfg, cluster_solve_kernel<N, XEMIT_ACC_SUB>, a, g, p);
        return cudaLaunchKernelEx(&cfg, cluster_solve_kernel<N, XEMIT_ADD>, a, g, p);
    }
}

}  // namespace dstk

#define IBPM_CLUSTER_DEFINE(N)                                                                       \
    cudaError_t cluster_solve_##N(const Geom& g, const DstPlan& p, const ClusterSolveArgs& a, int ns, \
                                  cudaStream_t st) {                                                 \
        return dstk::cluster_launch_t<N>(g, p, a, ns, st);                                           \
    }                                                                                                \
    cudaError_t cluster_attr_##N() { return dstk::cluster_attr_t<N>(); }

}  // namespace ibpm
