// Dense FP64 inverse of the Schur complement B on the device.  The reference
// forms inv(B) with LAPACK (src/fluid-operators/laplacian.jl:118); B built
// through the nested-grid vort2flux is not symmetric (its relative asymmetry is
// 1e-6 … 1e-4 on the configurations tested), so a Cholesky factor would change
// the solution well above round-off.  This is Gauss–Jordan elimination with
// partial pivoting (largest |pivot|, first index on ties) on [B | I].
#include "ibpm_internal.cuh"

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
