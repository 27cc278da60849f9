// Level chain of vort2flux! (src/fluid-operators/curl.jl:428-440) in spectral
// space.
//
// The reference telescopes from the coarsest level inwards,
//     ψ_l = Δ⁻¹ (Γ_l + apply_bc!(get_bc!(ψ_{l+1}))),   Δ⁻¹ = S D S,
// with S the 2-D DST-I and D = scale/Λ.  Δ⁻¹ is linear and the edge term b_l
// only touches the first/last rows and columns, so with Ĝ_l = S Γ_l (computed
// for every level at once):
//     Ŵ_l = D (Ĝ_l + S b_l),  ψ_l = S Ŵ_l,
// and S b_l is a sum of four outer products of 1-D DSTs of the edge vectors.
// get_bc! only samples ψ_{l+1} on rows jb = ny/4-1, jt = 3ny/4-1 and columns
// il = nx/4-1, ir = 3nx/4-1 (0-based), and
//     ψ(i, jb) = Σ_k Sx(i,k) v(k),  v(k) = Σ_m Sy(jb, m) Ŵ(k, m)
// (likewise for the other row and the two columns), so each chain step is one
// pass over the coarser spectral slab (four weighted sums, spread over a
// thread-block cluster and combined through distributed shared memory), then,
// in the cluster's first block, four 1-D DSTs to get the sampled rows/columns,
// get_bc!, and four 1-D DSTs of the edge vectors: the rank-4 image for the
// next level.
#pragma once

#include <cooperative_groups.h>

#include "dst_kernels.cuh"

namespace ibpm {
namespace ringk {

using dstk::ct_buf;
using dstk::ct_pad;
using dstk::ct_tp;
using dstk::ct_tw_count;
using dstk::dst_pair;
using dstk::gsync;
using dstk::stage_tables;

constexpr int CL_MAX = 16;        // blocks per cluster (one cluster per field): 16 or 8
constexpr int RING_THREADS = 256;
// Rows per pipeline chunk: two chunks of RCH rows of the spectral slab are in
// shared memory at a time (cp.async double buffering).
template <int NX>
__host__ __device__ constexpr int ring_rch() { return NX <= 512 ? 8 : (NX <= 768 ? 4 : 2); }
constexpr int RMAX = 128;         // rows of one block (n2 <= 1023 with 8 blocks)

template <int NX, int NY>
__host__ __device__ constexpr size_t ring_smem_bytes() {
    return dstk::tables_bytes<NX>() + dstk::tables_bytes<NY>() +
           (size_t)(ct_buf(NX) + ct_buf(NY)) * sizeof(double2) +
           (size_t)(4 * NX + 4 * NY) * sizeof(double) +   // finish vectors (block 0)
           (size_t)(2 * NX) * sizeof(double) +            // partial row-weighted sums of this block
           (size_t)(RMAX * 8) * sizeof(double) +          // per-row table values of the block
           (size_t)(2 * ring_rch<NX>() * NX) * sizeof(double) +  // chunk double buffer
           (size_t)(ring_rch<NX>() * (RING_THREADS / 32) * 2) * sizeof(double) + 64;
}

// One cluster of CL blocks per field (blockIdx.y = batch member).  Block b
// reduces spectral rows [b·rows, (b+1)·rows); the column sums meet in block 0
// through distributed shared memory, which then finishes the chain step.
template <int NX, int NY>
__global__ void __launch_bounds__(RING_THREADS) ring_kernel(RingArgs a, Geom g, DstPlan px, DstPlan py) {
    namespace cg = cooperative_groups;
    cg::cluster_group cluster = cg::this_cluster();
    const int CL = (int)cluster.num_blocks();
    extern __shared__ double2 smem2[];
    const int n1 = g.n1, n2 = g.n2, P = g.P;
    const int bt = blockIdx.y;
    const int rank = (int)cluster.block_rank();
    const int lc = a.lev + 1;  // the coarser level whose spectrum is read
    const double* __restrict__ T = a.T + a.tmap.off(bt * a.tmap.nlev + (lc - a.tmap.lev0));
    const double* __restrict__ rvc = a.r4.v + (long long)(bt * a.r4.mg + lc) * 4 * a.r4.len;
    const RingTabs& tb = a.tabs;

    // shared layout (identical in every block of the cluster)
    double2* twx = smem2;
    double* snx = reinterpret_cast<double*>(twx + ct_tw_count(NX));
    double2* twy = reinterpret_cast<double2*>(reinterpret_cast<char*>(smem2) + dstk::tables_bytes<NX>());
    double* sny = reinterpret_cast<double*>(twy + ct_tw_count(NY));
    double2* bufx = reinterpret_cast<double2*>(reinterpret_cast<char*>(smem2) + dstk::tables_bytes<NX>() +
                                               dstk::tables_bytes<NY>());
    double2* bufy = bufx + ct_buf(NX);
    double* rowb = reinterpret_cast<double*>(bufy + ct_buf(NY));  // [NX] v_jb → row jb → Sx bot
    double* rowt = rowb + NX;                                      // [NX] v_jt → row jt → Sx top
    double* edgx = rowt + NX;                                      // [2 NX] bot', top'
    double* coll = edgx + 2 * NX;                                  // [NY] u_il → column il → Sy left
    double* colr = coll + NY;                                      // [NY] u_ir → column ir → Sy right
    double* edgy = colr + NY;                                      // [2 NY] left', right'
    constexpr int RCH = ring_rch<NX>();
    double* vpart = edgy + 2 * NY;                                 // [2 NX] this block's column sums
    double* rtab = vpart + 2 * NX;                                 // [RMAX][8] per-row values
    double* chunk = rtab + RMAX * 8;                               // [2][RCH][NX] spectral rows
    double* red = chunk + 2 * RCH * NX;                            // [RCH][warps][2]

    if (rank == 0) {  // constant tables for phase 3, before the dependency wait
        stage_tables<NX>(twx, snx, px);
        stage_tables<NY>(twy, sny, py);
    }
    const int rows = (n2 + CL - 1) / CL;
    const int m_begin = rank * rows, m_end = min(n2, min(m_begin + rows, m_begin + RMAX));
    const int nrows = min(RMAX, max(0, m_end - m_begin));
    for (int r = threadIdx.x; r < nrows; r += RING_THREADS) {  // constant per-row tables
        const int m = m_begin + r;
        double* rt = rtab + r * 8;
        rt[0] = tb.cy[m]; rt[1] = tb.sy0[m]; rt[2] = tb.syN[m]; rt[5] = tb.syb[m]; rt[6] = tb.syt[m];
    }
    pdl_wait();
    pdl_trigger();
    for (int r = threadIdx.x; r < nrows; r += RING_THREADS) {  // edge image of the coarser level
        const int m = m_begin + r;
        rtab[r * 8 + 3] = rvc[2 * a.r4.len + m];
        rtab[r * 8 + 4] = rvc[3 * a.r4.len + m];
    }
    // cp.async one chunk (RCH rows starting at row mc) into buffer `buf`
    auto fetch = [&](int mc, int buf) {
        double* dst = chunk + buf * RCH * NX;
        for (int e = threadIdx.x; e < RCH * n1; e += RING_THREADS) {
            const int r = e / n1, k = e - r * n1;
            const int m = mc + r;
            if (m < m_end) cp_async8(dst + r * NX + k, T + (long long)m * P + k);
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };

    // ---- phase 1: this block's rows of Ŵ_lc, weighted sums
    constexpr int NC = (NX - 1 + RING_THREADS - 1) / RING_THREADS;
    constexpr int NW = RING_THREADS / 32;
    double vb[NC], vt[NC];
    double kx[NC][7];  // per column: cx, sxl, sxr, sx0, sxN, Sx bot, Sx top
#pragma unroll
    for (int c = 0; c < NC; ++c) {
        vb[c] = 0.0;
        vt[c] = 0.0;
        const int k = threadIdx.x + c * RING_THREADS;
        if (k < n1) {
            kx[c][0] = tb.cx[k]; kx[c][1] = tb.sxl[k]; kx[c][2] = tb.sxr[k];
            kx[c][3] = tb.sx0[k]; kx[c][4] = tb.sxN[k];
            kx[c][5] = rvc[k]; kx[c][6] = rvc[a.r4.len + k];
        }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double* ucl0 = cluster.map_shared_rank(coll, 0);  // block 0's column vectors
    double* ucr0 = cluster.map_shared_rank(colr, 0);
    cluster.sync();  // every block of the cluster runs before any remote store
    if (nrows > 0) fetch(m_begin, 0);
    int buf = 0;
    for (int mc = m_begin; mc < m_end; mc += RCH, buf ^= 1) {
        if (mc + RCH < m_end) {
            fetch(mc + RCH, buf ^ 1);  // next chunk in flight while this one is used
            asm volatile("cp.async.wait_group 1;" ::: "memory");
        } else {
            asm volatile("cp.async.wait_group 0;" ::: "memory");
        }
        __syncthreads();
        const double* cur = chunk + buf * RCH * NX;
#pragma unroll
        for (int r = 0; r < RCH; ++r) {
            const int m = mc + r;
            double rl = 0.0, rr = 0.0;
            if (m < m_end) {
                const double* rt = rtab + (m - m_begin) * 8;
                const double c2 = rt[0], y0 = rt[1], yN = rt[2], lf = rt[3], rtv = rt[4], wb = rt[5], wt = rt[6];
#pragma unroll
                for (int c = 0; c < NC; ++c) {
                    const int k = threadIdx.x + c * RING_THREADS;
                    if (k < n1) {
                        // Ŵ as the inverse y-pass forms it (dst_y_kernel, YMODE_INV)
                        const double lam = -2.0 * ((kx[c][0] + c2) - 2.0);
                        double v = cur[r * NX + k];
                        v = (((v + kx[c][5] * y0) + kx[c][6] * yN) + kx[c][3] * lf) + kx[c][4] * rtv;
                        const double w = (v * nr_rcp(lam)) * a.scale;
                        vb[c] += wb * w;
                        vt[c] += wt * w;
                        rl += kx[c][1] * w;
                        rr += kx[c][2] * w;
                    }
                }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                rl += __shfl_xor_sync(0xffffffffu, rl, o);
                rr += __shfl_xor_sync(0xffffffffu, rr, o);
            }
            if (lane == 0) {
                red[(r * NW + warp) * 2 + 0] = rl;
                red[(r * NW + warp) * 2 + 1] = rr;
            }
        }
        __syncthreads();  // red complete; the buffer just used may be refilled
        if (threadIdx.x < 2 * RCH) {  // row sums are complete: store them in block 0
            const int r = threadIdx.x >> 1, which = threadIdx.x & 1;
            const int m = mc + r;
            if (m < m_end) {
                double s = 0.0;
                for (int w = 0; w < NW; ++w) s += red[(r * NW + w) * 2 + which];
                (which ? ucr0 : ucl0)[m] = s;
            }
        }
    }
#pragma unroll
    for (int c = 0; c < NC; ++c) {
        const int k = threadIdx.x + c * RING_THREADS;
        if (k < n1) {
            vpart[k] = vb[c];
            vpart[NX + k] = vt[c];
        }
    }
    cluster.sync();
    // ---- phase 2: block b sums column slice b over the cluster (rank order)
    {
        const int cols = (n1 + CL - 1) / CL;
        const int k0 = rank * cols, k1 = min(n1, k0 + cols);
        double* vb0 = cluster.map_shared_rank(rowb, 0);
        double* vt0 = cluster.map_shared_rank(rowt, 0);
        for (int e = threadIdx.x; e < 2 * (k1 - k0); e += RING_THREADS) {
            const int which = e / (k1 - k0), k = k0 + e % (k1 - k0);
            double part[CL_MAX];
#pragma unroll
            for (int b = 0; b < CL_MAX; ++b)  // issue the remote loads together
                part[b] = b < CL ? cluster.map_shared_rank(vpart, b)[which * NX + k] : 0.0;
            double s = 0.0;
#pragma unroll
            for (int b = 0; b < CL_MAX; ++b)
                if (b < CL) s += part[b];
            (which ? vt0 : vb0)[k] = s;
        }
    }
    cluster.sync();
    if (rank != 0) return;

    // ---- phase 3 (block 0): sampled rows/columns, get_bc!, edge images
    cp_async_wait();
    __syncthreads();
    constexpr int TPX = ct_tp(NX), TPY = ct_tp(NY);
    static_assert(TPX + TPY <= RING_THREADS, "two transform groups must fit in one block");
    const int t = threadIdx.x;
    const bool gx = t < TPX, gy = t >= TPX && t < TPX + TPY;
    // sampled rows / columns of ψ_lc: ψ(i, jb) = Σ_k Sx(i,k) v(k)
    if (gx) {
        dst_pair<NX, TPX>(
            bufx, twx, snx, t, 0, [&](int i) { return make_double2(rowb[i], rowt[i]); },
            [&](int o, double2 v) { rowb[o] = v.x; rowt[o] = v.y; });
    } else if (gy) {
        dst_pair<NY, TPY>(
            bufy, twy, sny, t - TPX, 1, [&](int i) { return make_double2(coll[i], colr[i]); },
            [&](int o, double2 v) { coll[o] = v.x; colr[o] = v.y; });
    }
    __syncthreads();
    // get_bc! (mg-utils.jl:7-32) from the sampled lines, then the edge vectors
    // that apply_bc! adds at Γ index i (vertex i+1): bot'(i) = bot(i+1).
    auto samp = [](const double* line, int c0, int v) -> double {
        if ((v & 1) == 0) return line[c0 + (v >> 1)];
        const int ia = c0 + ((v + 1) >> 1);
        return 0.5 * (line[ia] + line[ia - 1]);
    };
    for (int i = t; i < n1; i += RING_THREADS) {
        edgx[i] = samp(rowb, g.nx / 4 - 1, i + 1);
        edgx[NX + i] = samp(rowt, g.nx / 4 - 1, i + 1);
    }
    for (int j = t; j < n2; j += RING_THREADS) {
        edgy[j] = samp(coll, g.ny / 4 - 1, j + 1);
        edgy[NY + j] = samp(colr, g.ny / 4 - 1, j + 1);
    }
    // the whole ψbc vector of level lev (vertices 0 … nx / 0 … ny), for the curl
    double* bcw = a.bcw + (long long)(bt * a.r4.mg + a.lev) * g.nbc;
    for (int v = t; v <= g.nx; v += RING_THREADS) {
        bcw[g.B + v] = samp(rowb, g.nx / 4 - 1, v);
        bcw[g.T + v] = samp(rowt, g.nx / 4 - 1, v);
    }
    for (int v = t; v <= g.ny; v += RING_THREADS) {
        bcw[g.L + v] = samp(coll, g.ny / 4 - 1, v);
        bcw[g.R + v] = samp(colr, g.ny / 4 - 1, v);
    }
    __syncthreads();
    double* rvf = a.r4w + (long long)(bt * a.r4.mg + a.lev) * 4 * a.r4.len;  // rank-4 image of lev
    if (gx) {
        dst_pair<NX, TPX>(
            bufx, twx, snx, t, 0, [&](int i) { return make_double2(edgx[i], edgx[NX + i]); },
            [&](int o, double2 v) { rvf[o] = v.x; rvf[a.r4.len + o] = v.y; });
    } else if (gy) {
        dst_pair<NY, TPY>(
            bufy, twy, sny, t - TPX, 1, [&](int j) { return make_double2(edgy[j], edgy[NY + j]); },
            [&](int o, double2 v) { rvf[2 * a.r4.len + o] = v.x; rvf[3 * a.r4.len + o] = v.y; });
    }
}

template <int NX, int NY>
struct RingCluster {
    static int size;  // blocks per cluster chosen at initialisation (16 if the GPU allows, else 8)
};
template <int NX, int NY>
int RingCluster<NX, NY>::size = 8;

template <int NX, int NY>
cudaError_t launch_ring_t(const Geom& g, const DstPlan& px, const DstPlan& py, const RingArgs& a, int nbatch,
                          cudaStream_t st) {
    const int cl = RingCluster<NX, NY>::size;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(cl, nbatch);
    cfg.blockDim = dim3(RING_THREADS);
    cfg.dynamicSmemBytes = ring_smem_bytes<NX, NY>();
    cfg.stream = st;
    cudaLaunchAttribute attr[2];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cl;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    attr[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[1].val.programmaticStreamSerializationAllowed = pdl_enabled() ? 1 : 0;
    cfg.attrs = attr;
    cfg.numAttrs = 2;
    return cudaLaunchKernelEx(&cfg, ring_kernel<NX, NY>, a, g, px, py);
}

template <int NX, int NY>
cudaError_t ring_attr_t() {
    cudaError_t e = cudaFuncSetAttribute(ring_kernel<NX, NY>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)ring_smem_bytes<NX, NY>());
    if (e != cudaSuccess) return e;
    // a 16-block cluster if this GPU can hold one, else the portable 8
    RingCluster<NX, NY>::size = 8;
    if (cudaFuncSetAttribute(ring_kernel<NX, NY>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) ==
        cudaSuccess) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(CL_MAX, 1);
        cfg.blockDim = dim3(RING_THREADS);
        cfg.dynamicSmemBytes = ring_smem_bytes<NX, NY>();
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = CL_MAX;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        int nclusters = 0;
        if (cudaOccupancyMaxActiveClusters(&nclusters, ring_kernel<NX, NY>, &cfg) == cudaSuccess && nclusters > 0)
            RingCluster<NX, NY>::size = CL_MAX;
    }
    cudaGetLastError();  // clear a refused attribute
    return cudaSuccess;
}

}  // namespace ringk

#define IBPM_RING_DEFINE(NX, NY)                                                                              \
    cudaError_t ring_##NX##_##NY(const Geom& g, const DstPlan& px, const DstPlan& py, const RingArgs& a, int nb, \
                                 cudaStream_t st) {                                                         \
        return ringk::launch_ring_t<NX, NY>(g, px, py, a, nb, st);                                          \
    }                                                                                                       \
    cudaError_t ring_attr_##NX##_##NY() { return ringk::ring_attr_t<NX, NY>(); }

}  // namespace ibpm
