// Boundary-transfer form of vort2flux! (src/fluid-operators/curl.jl:133-165):
// the edge-vector chain e_ℓ = get_bc!(Δ⁻¹Γ_{ℓ+1}) + R e_{ℓ+1} in a rank-k basis
// of R = get_bc! ∘ Δ⁻¹ ∘ apply_bc! (mg-utils.jl:7-60), and R's setup.  The
// transforms around it (the multi-level x- and y-passes, the line samples and
// the y-pass of the edge source) are in dst_kernels.cuh; the definitions in
// ibpm_internal.cuh.
#include "ibpm_internal.cuh"

#include <algorithm>
#include <cmath>
#include <thread>
#include <vector>

namespace ibpm {

namespace {

// get_bc! entry v (1 … n−1) of one edge from the n/2+1 line samples of the
// coarser level along it: even v copies a sample, odd v averages the two
// around it (mg-utils.jl:14-28).
template <class T>
__device__ __forceinline__ T edge_from_samples(const T* seg, int v) {
    if ((v & 1) == 0) return seg[v >> 1];
    return T(0.5) * (seg[(v + 1) >> 1] + seg[(v - 1) >> 1]);
}

// Entry m of g = get_bc!(level's samples) in the edge order bottom, top,
// left, right.
template <class T>
__device__ __forceinline__ T g_entry(const T* smp, const Geom& g, int m) {
    const int nx = g.nx, ny = g.ny, n1 = g.n1, n2 = g.n2;
    if (m < n1) return edge_from_samples(smp, m + 1);
    if (m < 2 * n1) return edge_from_samples(smp + nx / 2 + 1, m - n1 + 1);
    if (m < 2 * n1 + n2) return edge_from_samples(smp + nx + 2, m - 2 * n1 + 1);
    return edge_from_samples(smp + nx + 2 + ny / 2 + 1, m - 2 * n1 - n2 + 1);
}

constexpr int kMaxLev = 8;

// p_ℓ[r] = Σ_s Ws[r, s] smp_{ℓ+1}[s] for every level ℓ = 0 … mg−2, with
// Ws = W A_s the projection folded with get_bc!'s averaging of the samples
// (A_s: g = A_s · samples).  One block per row r of Ws (read once for all
// levels): its threads take s in a fixed order, the loads of eight steps
// issued together, then a fixed-order reduction over the block.
template <class T>
__global__ void __launch_bounds__(256) bt_project_kernel(const T* __restrict__ Ws, const T* __restrict__ samples,
                                                         T* p, int k, int kp, Geom g) {
    __shared__ T red[8 * kMaxLev];
    pdl_wait();
    pdl_trigger();
    const int L = g.mg - 1;
    const int sl = g.nx + g.ny + 4, sp = (sl + 3) & ~3;
    const int r = blockIdx.x, tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    samples += (long long)blockIdx.y * g.mg * sl;   // simulation blockIdx.y of a batch group
    p += (long long)blockIdx.y * L * kp;
    T acc[kMaxLev];
#pragma unroll
    for (int l = 0; l < kMaxLev; ++l) acc[l] = T(0);
    const T* row = Ws + (long long)r * sp;
#pragma unroll 8
    for (int s = tid; s < sl; s += 256) {
        const T wv = __ldg(&row[s]);
#pragma unroll
        for (int l = 0; l < kMaxLev; ++l)
            if (l < L) acc[l] += wv * __ldg(&samples[(long long)(l + 1) * sl + s]);
    }
#pragma unroll
    for (int l = 0; l < kMaxLev; ++l) {
        if (l < L) {
            T v = acc[l];
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
            if (lane == 0) red[w * kMaxLev + l] = v;
        }
    }
    __syncthreads();
    if (tid < L && r < k) {
        T v = T(0);
#pragma unroll
        for (int q = 0; q < 8; ++q) v += red[q * kMaxLev + tid];
        p[(long long)tid * kp + r] = v;
    }
}

// e_ℓ[i] = g_ℓ[i] + Σ_{m=0}^{mg−3−ℓ} U_m[i, :] · p_{ℓ+1+m}: one warp per row i,
// lanes over the rank index in a fixed order.  The (m, rank) steps run as one
// flat loop, so the loads of eight steps (of all U_m) are issued together; the
// projections are staged in shared memory.
template <class T>
__global__ void __launch_bounds__(256) bt_expand_kernel(const T* __restrict__ U, const T* __restrict__ samples,
                                                        const T* __restrict__ p, T* e, int k, int kp, Geom g) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* ps = reinterpret_cast<T*>(smem_raw);
    pdl_wait();
    pdl_trigger();
    const int nE = 2 * g.n1 + 2 * g.n2, ep = (nE + 3) & ~3, L = g.mg - 1;
    const int sl = g.nx + g.ny + 4;
    samples += (long long)blockIdx.y * g.mg * sl;   // simulation blockIdx.y of a batch group
    p += (long long)blockIdx.y * L * kp;
    e += (long long)blockIdx.y * g.mg * ep;
    for (int t = threadIdx.x; t < L * kp; t += blockDim.x) ps[t] = p[t];
    __syncthreads();
    const int i = blockIdx.x * 8 + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (i >= nE) return;
    T acc[kMaxLev];
#pragma unroll
    for (int l = 0; l < kMaxLev; ++l) acc[l] = T(0);
    const int nt = (k + 31) >> 5, steps = (g.mg - 2) * nt;
    int m = 0, t = 0;
#pragma unroll 8
    for (int j = 0; j < steps; ++j) {
        const int r = lane + 32 * t;
        const T u = r < k ? __ldg(&U[((long long)m * nE + i) * kp + r]) : T(0);
        const int rr = r < k ? r : 0;
#pragma unroll
        for (int l = 0; l < kMaxLev; ++l)
            if (l + m + 1 < L) acc[l] += u * ps[(l + 1 + m) * kp + rr];
        if (++t == nt) { t = 0; ++m; }
    }
#pragma unroll
    for (int l = 0; l < kMaxLev; ++l) {
        if (l < L) {
            T v = acc[l];
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
            if (lane == 0) e[(long long)l * ep + i] = g_entry(samples + (long long)(l + 1) * sl, g, i) + v;
        }
    }
}

// The grid point where edge entry k of apply_bc! adds its value (0-based).
__device__ __forceinline__ void edge_point(const Geom& g, int k, int& i, int& j) {
    if (k < g.n1) { i = k; j = 0; }
    else if (k < 2 * g.n1) { i = k - g.n1; j = g.n2 - 1; }
    else if (k < 2 * g.n1 + g.n2) { i = 0; j = k - 2 * g.n1; }
    else { i = g.n1 - 1; j = k - 2 * g.n1 - g.n2; }
}

__global__ void bt_unit_src_kernel(Geom g, int c0, int ncol, double* G, long long bstride) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= ncol) return;
    int i, j;
    edge_point(g, c0 + b, i, j);
    G[(long long)b * bstride + (long long)j * g.P + i] = 1.0;
}

// R[m, c0 + b] = get_bc! entry m of the solve in slab b.
__global__ void bt_gather_kernel(Geom g, int c0, int ncol, const double* psi, long long bstride, double* R) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    const int b = blockIdx.y;
    const int nE = 2 * g.n1 + 2 * g.n2, ep = (nE + 3) & ~3;
    if (m >= nE || b >= ncol) return;
    CoarseBC cb;
    cb.rc = psi + (long long)b * bstride; cb.P = g.P; cb.nx = g.nx; cb.ny = g.ny;
    double v;
    if (m < g.n1) v = cb.bot(m + 1);
    else if (m < 2 * g.n1) v = cb.top(m - g.n1 + 1);
    else if (m < 2 * g.n1 + g.n2) v = cb.left(m - 2 * g.n1 + 1);
    else v = cb.right(m - 2 * g.n1 - g.n2 + 1);
    R[(long long)m * ep + c0 + b] = v;
}

// Run f(t0, t1) over [0, n) split across the host's threads.
template <class F>
void parallel_for(int n, F f) {
    const int nt = std::max(1, std::min<int>(16, (int)std::thread::hardware_concurrency()));
    if (nt == 1 || n < 64) { f(0, n); return; }
    std::vector<std::thread> th;
    const int chunk = (n + nt - 1) / nt;
    for (int t = 0; t < nt; ++t) {
        const int a = t * chunk, b = std::min(n, a + chunk);
        if (a < b) th.emplace_back(f, a, b);
    }
    for (auto& x : th) x.join();
}

}  // namespace

// Rank-k basis of R (nE × nE, row-major with pitch ep): Gram–Schmidt with
// column pivoting (Businger & Golub, 1965), each new direction orthogonalised
// twice against the earlier ones, stopped at the first residual column norm
// below tol × R's largest column norm.  Then W = Qᵀ R, M = W Q and
// U_m = Q M^m for m < nmat.  Every step has a fixed order, so the factors
// do not depend on the thread count.
int bt_lowrank(const std::vector<double>& R, int nx_, int ny_, int nmat, double tol, int kmax, BtLowRank& out) {
    const int nE = 2 * (nx_ - 1) + 2 * (ny_ - 1), ep = (nE + 3) & ~3;
    std::vector<double> A((size_t)nE * nE);  // column-major residual columns
    parallel_for(nE, [&](int j0, int j1) {
        for (int j = j0; j < j1; ++j)
            for (int i = 0; i < nE; ++i) A[(size_t)j * nE + i] = R[(size_t)i * ep + j];
    });
    std::vector<double> n2(nE);
    auto norms = [&](int j0, int j1) {
        for (int j = j0; j < j1; ++j) {
            double s = 0.0;
            const double* a = &A[(size_t)j * nE];
            for (int i = 0; i < nE; ++i) s += a[i] * a[i];
            n2[j] = s;
        }
    };
    parallel_for(nE, norms);
    std::vector<std::vector<double>> Q;
    double nmax = 0.0;
    for (int r = 0; r < kmax; ++r) {
        int p = 0;
        for (int j = 1; j < nE; ++j)
            if (n2[j] > n2[p]) p = j;
        const double np = std::sqrt(n2[p]);
        if (r == 0) nmax = np;
        if (!(np > tol * nmax)) break;
        std::vector<double> q(A.begin() + (size_t)p * nE, A.begin() + (size_t)(p + 1) * nE);
        for (int pass = 0; pass < 2; ++pass) {
            for (const auto& qs : Q) {
                double d = 0.0;
                for (int i = 0; i < nE; ++i) d += qs[i] * q[i];
                for (int i = 0; i < nE; ++i) q[i] -= d * qs[i];
            }
            double s = 0.0;
            for (int i = 0; i < nE; ++i) s += q[i] * q[i];
            s = 1.0 / std::sqrt(s);
            for (int i = 0; i < nE; ++i) q[i] *= s;
        }
        parallel_for(nE, [&](int j0, int j1) {
            for (int j = j0; j < j1; ++j) {
                double* a = &A[(size_t)j * nE];
                double t = 0.0;
                for (int i = 0; i < nE; ++i) t += q[i] * a[i];
                double s = 0.0;
                for (int i = 0; i < nE; ++i) {
                    a[i] -= t * q[i];
                    s += a[i] * a[i];
                }
                n2[j] = s;
            }
        });
        Q.push_back(std::move(q));
    }
    const int k = (int)Q.size();
    if (k == 0 || k >= kmax) return -1;
    const int kp = (k + 3) & ~3;
    out.k = k;
    out.kp = kp;
    out.W.assign((size_t)k * ep, 0.0);
    parallel_for(k, [&](int r0, int r1) {
        for (int r = r0; r < r1; ++r) {
            double* w = &out.W[(size_t)r * ep];
            for (int i = 0; i < nE; ++i) {
                const double qi = Q[r][i];
                const double* ri = &R[(size_t)i * ep];
                for (int j = 0; j < nE; ++j) w[j] += qi * ri[j];
            }
        }
    });
    // Ws = W A_s: edge entry m (get_bc! vertex v = m' + 1 of its edge) is
    // sample v/2 of the edge's line (v even) or the mean of samples (v±1)/2
    const int sl = nx_ + ny_ + 4, sp = (sl + 3) & ~3;
    out.Ws.assign((size_t)k * sp, 0.0);
    auto add_edge = [&](double* ws, const double* w, int off, int n1e, int seg) {
        for (int mm = 0; mm < n1e; ++mm) {
            const int v = mm + 1;
            const double wv = w[off + mm];
            if ((v & 1) == 0) ws[seg + v / 2] += wv;
            else {
                ws[seg + (v + 1) / 2] += 0.5 * wv;
                ws[seg + (v - 1) / 2] += 0.5 * wv;
            }
        }
    };
    parallel_for(k, [&](int r0, int r1) {
        for (int r = r0; r < r1; ++r) {
            double* ws = &out.Ws[(size_t)r * sp];
            const double* w = &out.W[(size_t)r * ep];
            const int n1 = nx_ - 1, n2 = ny_ - 1;
            add_edge(ws, w, 0, n1, 0);                                  // bottom: row samples at 0
            add_edge(ws, w, n1, n1, nx_ / 2 + 1);                       // top
            add_edge(ws, w, 2 * n1, n2, nx_ + 2);                       // left: column samples
            add_edge(ws, w, 2 * n1 + n2, n2, nx_ + 2 + ny_ / 2 + 1);    // right
        }
    });
    out.sp = sp;
    std::vector<double> M((size_t)k * k);
    parallel_for(k, [&](int a0, int a1) {
        for (int a = a0; a < a1; ++a)
            for (int b = 0; b < k; ++b) {
                double s = 0.0;
                for (int j = 0; j < nE; ++j) s += out.W[(size_t)a * ep + j] * Q[b][j];
                M[(size_t)a * k + b] = s;
            }
    });
    out.U.assign((size_t)nmat * nE * kp, 0.0);
    for (int m = 0; m < nmat; ++m) {
        double* Um = &out.U[(size_t)m * nE * kp];
        if (m == 0) {
            for (int i = 0; i < nE; ++i)
                for (int r = 0; r < k; ++r) Um[(size_t)i * kp + r] = Q[r][i];
        } else {
            const double* Up = &out.U[(size_t)(m - 1) * nE * kp];
            parallel_for(nE, [&](int i0, int i1) {
                for (int i = i0; i < i1; ++i)
                    for (int b = 0; b < k; ++b) {
                        double s = 0.0;
                        for (int a = 0; a < k; ++a) s += Up[(size_t)i * kp + a] * M[(size_t)a * k + b];
                        Um[(size_t)i * kp + b] = s;
                    }
            });
        }
    }
    return 0;
}

cudaError_t launch_bt_project(const Geom& g, const BtChainArgs& a, cudaStream_t st) {
    dim3 grid(a.k, std::max(1, a.nsim));
    return launch_k(bt_project_kernel<double>, grid, dim3(256), 0, st, a.W, a.samples, a.p, a.k, a.kp, g);
}

cudaError_t launch_bt_expand(const Geom& g, const BtChainArgs& a, cudaStream_t st) {
    dim3 grid((bt_edge_len(g) + 7) / 8, std::max(1, a.nsim));
    const size_t smem = (size_t)(g.mg - 1) * a.kp * sizeof(double);
    return launch_k(bt_expand_kernel<double>, grid, dim3(256), smem, st, a.U, a.samples,
                    static_cast<const double*>(a.p), a.e, a.k, a.kp, g);
}

cudaError_t launch_bt_unit_src(const Geom& g, int c0, int ncol, double* G, long long bstride, cudaStream_t st) {
    bt_unit_src_kernel<<<(ncol + 127) / 128, 128, 0, st>>>(g, c0, ncol, G, bstride);
    return cudaGetLastError();
}

cudaError_t launch_bt_gather(const Geom& g, int c0, int ncol, const double* psi, long long bstride, double* R,
                             cudaStream_t st) {
    dim3 grid((bt_edge_len(g) + 127) / 128, ncol);
    bt_gather_kernel<<<grid, 128, 0, st>>>(g, c0, ncol, psi, bstride, R);
    return cudaGetLastError();
}

}  // namespace ibpm
