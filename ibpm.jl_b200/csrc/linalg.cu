// Dense FP64 inverse of the Schur complement B on the device.  The reference
// forms inv(B) with LAPACK (src/fluid-operators/laplacian.jl:118); B built
// through the nested-grid vort2flux is not symmetric (its relative asymmetry is
// 1e-6 … 1e-4 on the configurations tested), so a Cholesky factor would change
// the solution well above round-off.  This is Gauss–Jordan elimination with
// partial pivoting (largest |pivot|, first index on ties) on [B | I].
#include "ibpm_internal.cuh"

#include <algorithm>

namespace ibpm {

// One block: choose the pivot of column c, swap it into row c, normalise row c
// and save the multipliers of column c for the elimination kernel.
__global__ void gj_pivot_kernel(double* aug, int n, int c, double* fcol, int* info) {
    __shared__ double bv[1024];
    __shared__ int bi[1024];
    const int n2 = 2 * n;
    double best = -1.0;
    int bidx = n;
    for (int r = c + threadIdx.x; r < n; r += blockDim.x) {
        const double v = fabs(aug[(long long)r * n2 + c]);
        if (v > best) { best = v; bidx = r; }
    }
    bv[threadIdx.x] = best;
    bi[threadIdx.x] = bidx;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            const double o = bv[threadIdx.x + s];
            const int oi = bi[threadIdx.x + s];
            if (o > bv[threadIdx.x] || (o == bv[threadIdx.x] && oi < bi[threadIdx.x])) {
                bv[threadIdx.x] = o;
                bi[threadIdx.x] = oi;
            }
        }
        __syncthreads();
    }
    const int p = bi[0];
    if (p >= n || bv[0] == 0.0) {
        if (threadIdx.x == 0 && *info == 0) *info = c + 1;
        return;
    }
    if (p != c) {
        for (int col = threadIdx.x; col < n2; col += blockDim.x) {
            const double t = aug[(long long)c * n2 + col];
            aug[(long long)c * n2 + col] = aug[(long long)p * n2 + col];
            aug[(long long)p * n2 + col] = t;
        }
    }
    __syncthreads();
    const double piv = aug[(long long)c * n2 + c];
    __syncthreads();
    for (int col = threadIdx.x; col < n2; col += blockDim.x) aug[(long long)c * n2 + col] /= piv;
    for (int r = threadIdx.x; r < n; r += blockDim.x) fcol[r] = (r == c) ? 0.0 : aug[(long long)r * n2 + c];
}

// aug[r][col] -= fcol[r] * aug[c][col] for every row r ≠ c.
__global__ void gj_elim_kernel(double* aug, int n, int c, const double* __restrict__ fcol, const int* info) {
    if (*info) return;
    const int n2 = 2 * n;
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    const int r = blockIdx.y;
    if (col >= n2 || r == c) return;
    const double f = fcol[r];
    if (f == 0.0) return;
    aug[(long long)r * n2 + col] -= f * aug[(long long)c * n2 + col];
}

__global__ void gj_setup_kernel(const double* A, double* aug, int n) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long tot = (long long)n * 2 * n;
    if (t >= tot) return;
    const int r = (int)(t / (2 * n)), col = (int)(t % (2 * n));
    aug[t] = (col < n) ? A[(long long)r * n + col] : (col - n == r ? 1.0 : 0.0);
}

__global__ void gj_extract_kernel(const double* aug, double* A, int n) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)n * n) return;
    const int r = (int)(t / n), col = (int)(t % n);
    A[t] = aug[(long long)r * 2 * n + n + col];
}

// The same elimination in ONE block with [B | I] in shared memory, for n up
// to kGjSmemMax: the pivot search, row swap, normalisation and elimination of
// each column are separated by block barriers instead of kernel boundaries
// (2n + 2 launches become one).  Every element sees the same operations in
// the same order as above (largest |pivot|, first index on ties; row c
// divided by the pivot; aug[r][col] -= f·aug[c][col] with f saved before the
// column is eliminated), so the result is the multi-launch one.
constexpr int kGjThreads = 1024;
constexpr int kGjSmemMax = 112;   // 2·112²·8 B + 112·8 B = 201 KB of shared memory
static size_t gj_smem_bytes(int n) { return ((size_t)2 * n * n + n) * sizeof(double); }

__global__ void __launch_bounds__(kGjThreads, 1) gj_inverse_smem_kernel(double* A, int n, int* info) {
    extern __shared__ __align__(16) double gsm[];
    __shared__ double wv[kGjThreads / 32];
    __shared__ int wi[kGjThreads / 32];
    __shared__ int s_piv;
    const int n2 = 2 * n;
    double* aug = gsm;
    double* fcol = gsm + (size_t)n * n2;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int t = tid; t < n * n2; t += kGjThreads) {
        const int r = t / n2, col = t - r * n2;
        aug[t] = (col < n) ? A[(long long)r * n + col] : (col - n == r ? 1.0 : 0.0);
    }
    __syncthreads();
    int bad = 0;
    for (int c = 0; c < n; ++c) {
        // pivot: the largest |aug[r][c]|, r >= c, the smallest r among equals
        double best = -1.0;
        int bidx = n;
        for (int r = c + tid; r < n; r += kGjThreads) {
            const double v = fabs(aug[r * n2 + c]);
            if (v > best) { best = v; bidx = r; }
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            const double o = __shfl_down_sync(0xffffffffu, best, off);
            const int oi = __shfl_down_sync(0xffffffffu, bidx, off);
            if (o > best || (o == best && oi < bidx)) { best = o; bidx = oi; }
        }
        if (lane == 0) { wv[warp] = best; wi[warp] = bidx; }
        __syncthreads();
        if (warp == 0) {
            best = wv[lane];
            bidx = wi[lane];
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) {
                const double o = __shfl_down_sync(0xffffffffu, best, off);
                const int oi = __shfl_down_sync(0xffffffffu, bidx, off);
                if (o > best || (o == best && oi < bidx)) { best = o; bidx = oi; }
            }
            if (lane == 0) s_piv = (bidx >= n || best == 0.0) ? -1 : bidx;
        }
        __syncthreads();
        const int p = s_piv;
        if (p < 0) { bad = c + 1; break; }     // every thread reads the same p
        if (p != c) {
            for (int col = tid; col < n2; col += kGjThreads) {
                const double t = aug[c * n2 + col];
                aug[c * n2 + col] = aug[p * n2 + col];
                aug[p * n2 + col] = t;
            }
        }
        __syncthreads();
        const double piv = aug[c * n2 + c];
        __syncthreads();
        for (int col = tid; col < n2; col += kGjThreads) aug[c * n2 + col] /= piv;
        for (int r = tid; r < n; r += kGjThreads) fcol[r] = (r == c) ? 0.0 : aug[r * n2 + c];
        __syncthreads();
        for (int t = tid; t < n * n2; t += kGjThreads) {
            const int r = t / n2, col = t - r * n2;
            if (r == c) continue;
            const double f = fcol[r];
            if (f == 0.0) continue;
            aug[r * n2 + col] -= f * aug[c * n2 + col];
        }
        __syncthreads();
    }
    for (int t = tid; t < n * n; t += kGjThreads) {
        const int r = t / n, col = t - r * n;
        A[t] = aug[r * n2 + n + col];
    }
    if (tid == 0) *info = bad;
}

// ---------------------------------------------------------------------------
// Blocked Gauss–Jordan for large n (the Schur complement of many body points):
// the elimination of a panel J of nb columns is a matrix T with T P = E_J
// (P the panel after its row swaps, E_J the unit columns J) that differs from
// I only in columns J, T = I + X S_J, so X = (E_J − P) · P[J, :]⁻¹ and the
// whole augmented matrix takes the panel's elimination as ONE rank-nb update
//     aug ← aug + X · aug[J, :]        (after the panel's row swaps).
// The panel's pivots are those of the column-by-column elimination: the
// panel is eliminated column by column first (largest |pivot|, first index on
// ties), on its own copy, to find them.  Columns left of the panel are never
// read again and are not updated.
// ---------------------------------------------------------------------------
constexpr int kGjPanel = 64;
constexpr int kGjBlockedMin = 513;   // from this n on the blocked form

__global__ void gjb_copy_panel(const double* aug, int n, int j0, int w, double* P, double* P0) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)n * w) return;
    const int r = (int)(t / w), c = (int)(t % w);
    const double v = aug[(long long)r * 2 * n + j0 + c];
    P[t] = v;
    P0[t] = v;
}

// Pivot of panel column c (global j0 + c): swap it into row j0 + c of P,
// normalise that row and keep the multipliers.
__global__ void gjb_panel_pivot(double* P, int n, int w, int j0, int c, double* fcol, int* piv, int* info) {
    __shared__ double bv[1024];
    __shared__ int bi[1024];
    const int pr = j0 + c;
    double best = -1.0;
    int bidx = n;
    for (int r = pr + threadIdx.x; r < n; r += blockDim.x) {
        const double v = fabs(P[(long long)r * w + c]);
        if (v > best) { best = v; bidx = r; }
    }
    bv[threadIdx.x] = best;
    bi[threadIdx.x] = bidx;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            const double o = bv[threadIdx.x + s];
            const int oi = bi[threadIdx.x + s];
            if (o > bv[threadIdx.x] || (o == bv[threadIdx.x] && oi < bi[threadIdx.x])) {
                bv[threadIdx.x] = o;
                bi[threadIdx.x] = oi;
            }
        }
        __syncthreads();
    }
    const int p = bi[0];
    if (p >= n || bv[0] == 0.0) {
        if (threadIdx.x == 0) {
            if (*info == 0) *info = pr + 1;
            piv[c] = pr;
        }
        return;
    }
    if (threadIdx.x == 0) piv[c] = p;
    if (p != pr) {
        for (int col = threadIdx.x; col < w; col += blockDim.x) {
            const double t = P[(long long)pr * w + col];
            P[(long long)pr * w + col] = P[(long long)p * w + col];
            P[(long long)p * w + col] = t;
        }
    }
    __syncthreads();
    const double pv = P[(long long)pr * w + c];
    __syncthreads();
    for (int col = threadIdx.x; col < w; col += blockDim.x) P[(long long)pr * w + col] /= pv;
    for (int r = threadIdx.x; r < n; r += blockDim.x) fcol[r] = (r == pr) ? 0.0 : P[(long long)r * w + c];
}

__global__ void gjb_panel_elim(double* P, int n, int w, int j0, int c, const double* __restrict__ fcol,
                               const int* info) {
    if (*info) return;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)n * w) return;
    const int r = (int)(t / w), col = (int)(t % w);
    if (r == j0 + c) return;
    const double f = fcol[r];
    if (f != 0.0) P[t] -= f * P[(long long)(j0 + c) * w + col];
}

// The panel's row swaps, in order, on the original panel P0 and on the
// columns [j0 + w, 2n) of aug; then D = P0[J, :] (w × w) and the row block
// Rb = aug[J, j0 + w : 2n].
__global__ void gjb_swaps(double* aug, int n, int j0, int w, const int* piv, double* P0, double* D, double* Rb) {
    const int n2 = 2 * n, c1 = j0 + w;
    for (int c = 0; c < w; ++c) {
        const int a = j0 + c, b = piv[c];
        if (a != b) {
            for (int col = c1 + threadIdx.x; col < n2; col += blockDim.x) {
                const double t = aug[(long long)a * n2 + col];
                aug[(long long)a * n2 + col] = aug[(long long)b * n2 + col];
                aug[(long long)b * n2 + col] = t;
            }
            for (int col = threadIdx.x; col < w; col += blockDim.x) {
                const double t = P0[(long long)a * w + col];
                P0[(long long)a * w + col] = P0[(long long)b * w + col];
                P0[(long long)b * w + col] = t;
            }
        }
        __syncthreads();
    }
    for (int t = threadIdx.x; t < w * w; t += blockDim.x) D[t] = P0[(long long)(j0 + t / w) * w + t % w];
    const int m = n2 - c1;
    for (long long t = threadIdx.x; t < (long long)w * m; t += blockDim.x) {
        const int r = (int)(t / m), col = (int)(t % m);
        Rb[t] = aug[(long long)(j0 + r) * n2 + c1 + col];
    }
}

// X = (E_J − P0) · Dinv   (n × w)
__global__ void gjb_x(const double* P0, const double* __restrict__ Dinv, int n, int w, int j0, double* X) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)n * w) return;
    const int r = (int)(t / w), c = (int)(t % w);
    double s = 0.0;
    for (int k = 0; k < w; ++k) {
        const double e = ((r - j0) == k) ? 1.0 : 0.0;
        s += (e - P0[(long long)r * w + k]) * Dinv[k * w + c];
    }
    X[t] = s;
}

// aug[:, j0 + w : 2n] += X · Rb, 64×64 tiles of C per block, k in chunks of 32.
__global__ void __launch_bounds__(256) gjb_update(double* aug, int n, int j0, int w, const double* __restrict__ X,
                                                  const double* __restrict__ Rb) {
    __shared__ double Xs[64][33];
    __shared__ double Rs[32][65];
    const int n2 = 2 * n, c1 = j0 + w, m = n2 - c1;
    const int r0 = blockIdx.y * 64, col0 = blockIdx.x * 64;
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;   // 16 × 16 threads, 4 × 4 outputs each
    double acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] = 0.0;
    for (int k0 = 0; k0 < w; k0 += 32) {
        for (int t = threadIdx.x; t < 64 * 32; t += 256) {
            const int rr = t / 32, kk = t % 32;
            Xs[rr][kk] = (r0 + rr < n && k0 + kk < w) ? X[(long long)(r0 + rr) * w + k0 + kk] : 0.0;
            const int k2 = t / 64, cc = t % 64;
            Rs[k2][cc] = (k0 + k2 < w && col0 + cc < m) ? Rb[(long long)(k0 + k2) * m + col0 + cc] : 0.0;
        }
        __syncthreads();
#pragma unroll 8
        for (int kk = 0; kk < 32; ++kk) {
            double xa[4], rb[4];
#pragma unroll
            for (int a = 0; a < 4; ++a) xa[a] = Xs[ty * 4 + a][kk];
#pragma unroll
            for (int b = 0; b < 4; ++b) rb[b] = Rs[kk][tx + 16 * b];
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b) acc[a][b] = fma(xa[a], rb[b], acc[a][b]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        const int r = r0 + ty * 4 + a;
        if (r >= n) continue;
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            const int col = col0 + tx + 16 * b;
            if (col < m) aug[(long long)r * n2 + c1 + col] += acc[a][b];
        }
    }
}

size_t gj_work_doubles(int n) {
    const size_t base = (size_t)2 * n * n + 2 * (size_t)n;
    if (n < kGjBlockedMin) return base;
    const size_t w = kGjPanel;
    // P, P0, X (n × w each), D (w × w), Rb (w × 2n), piv (w + 1 ints)
    return base + 3 * (size_t)n * w + w * w + w * 2 * (size_t)n + w;
}

static cudaError_t gj_inverse_blocked(double* A, int n, double* work, int* info, cudaStream_t st) {
    double* aug = work;
    double* fcol = work + (size_t)2 * n * n;
    const int W = kGjPanel;
    double* P = fcol + 2 * (size_t)n;
    double* P0 = P + (size_t)n * W;
    double* X = P0 + (size_t)n * W;
    double* D = X + (size_t)n * W;
    double* Rb = D + (size_t)W * W;
    int* piv = reinterpret_cast<int*>(Rb + (size_t)W * 2 * n);
    int* dinfo = piv + W;   // status of the panel blocks' inverses (never singular after pivoting)
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaError_t e = cudaStreamIsCapturing(st, &cs);
    if (e == cudaSuccess && cs == cudaStreamCaptureStatusNone)
        e = cudaFuncSetAttribute(gj_inverse_smem_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)gj_smem_bytes(kGjSmemMax));
    if (e == cudaSuccess) e = cudaMemsetAsync(info, 0, sizeof(int), st);
    if (e != cudaSuccess) return e;
    const long long tot = (long long)2 * n * n;
    gj_setup_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(A, aug, n);
    for (int j0 = 0; j0 < n; j0 += W) {
        const int w = std::min(W, n - j0);
        const unsigned gp = (unsigned)(((long long)n * w + 255) / 256);
        gjb_copy_panel<<<gp, 256, 0, st>>>(aug, n, j0, w, P, P0);
        for (int c = 0; c < w; ++c) {
            gjb_panel_pivot<<<1, 1024, 0, st>>>(P, n, w, j0, c, fcol, piv, info);
            gjb_panel_elim<<<gp, 256, 0, st>>>(P, n, w, j0, c, fcol, info);
        }
        gjb_swaps<<<1, 1024, 0, st>>>(aug, n, j0, w, piv, P0, D, Rb);
        gj_inverse_smem_kernel<<<1, kGjThreads, gj_smem_bytes(w), st>>>(D, w, dinfo);
        gjb_x<<<gp, 256, 0, st>>>(P0, D, n, w, j0, X);
        const int m = 2 * n - (j0 + w);
        if (m > 0) {
            dim3 grid((m + 63) / 64, (n + 63) / 64);
            gjb_update<<<grid, 256, 0, st>>>(aug, n, j0, w, X, Rb);
        }
    }
    gj_extract_kernel<<<(unsigned)(((long long)n * n + 255) / 256), 256, 0, st>>>(aug, A, n);
    return cudaGetLastError();
}

cudaError_t launch_gj_inverse(double* A, int n, double* work, int* info, cudaStream_t st) {
    if (n >= 1 && n <= kGjSmemMax) {
        // the shared-memory opt-in is a function attribute: set outside stream
        // capture (the handle's setup inverts B before any capture)
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        cudaError_t e = cudaStreamIsCapturing(st, &cs);
        if (e != cudaSuccess) return e;
        if (cs == cudaStreamCaptureStatusNone) {
            e = cudaFuncSetAttribute(gj_inverse_smem_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)gj_smem_bytes(kGjSmemMax));
            if (e != cudaSuccess) return e;
        }
        gj_inverse_smem_kernel<<<1, kGjThreads, gj_smem_bytes(n), st>>>(A, n, info);
        return cudaGetLastError();
    }
    if (n >= kGjBlockedMin) return gj_inverse_blocked(A, n, work, info, st);
    double* aug = work;
    double* fcol = work + (size_t)2 * n * n;
    cudaMemsetAsync(info, 0, sizeof(int), st);
    const long long tot = (long long)2 * n * n;
    gj_setup_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(A, aug, n);
    for (int c = 0; c < n; ++c) {
        gj_pivot_kernel<<<1, 1024, 0, st>>>(aug, n, c, fcol, info);
        dim3 grid((2 * n + 255) / 256, n);
        gj_elim_kernel<<<grid, 256, 0, st>>>(aug, n, c, fcol, info);
    }
    gj_extract_kernel<<<(unsigned)(((long long)n * n + 255) / 256), 256, 0, st>>>(aug, A, n);
    return cudaGetLastError();
}

}  // namespace ibpm
