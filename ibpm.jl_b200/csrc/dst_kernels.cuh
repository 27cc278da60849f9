// Batched 2-D DST-I (FFTW RODFT00, unnormalised) for the Poisson-type solves of
// the IBPM step: x = S((S b) ./ M .* scale), S the 2-D DST-I
// (src/fluid-operators/dst-inversion.jl:39-50, laplacian.jl:24-76).
//
// A 1-D DST-I of length n = N-1,  Y_k = 2 Σ_m f_m sin(π m k / N)  (f_m = X_{m-1}),
// is computed for TWO real lines at once (f = a + i b) with one complex FFT of
// length N:
//   y_m = sin(πm/N)(f_m + f_{N-m}) + ½(f_m − f_{N-m}),   y_0 = 0
//   Z   = Σ_m y_m e^{+2πi mk/N}
//   Y_{2k-1} = −i (Z_k − Z_{N-k})                       (k = 1 … N/2−1)
//   Y_{2k}   = Z_0 + Σ_{k'=1..k} (Z_{k'} + Z_{N-k'})    (k = 0 … N/2−1)
// (the sine transform through a half-length real FFT: the symmetric part of y
// carries the odd harmonics as a running sum, the antisymmetric part the even
// ones).  Re Y is line a, Im Y is line b.
//
// The FFT is a mixed-radix Stockham transform, run in place in shared memory
// by one "group" of TP threads (at least one warp): each stage reads all its
// inputs into registers, synchronises the group, then writes.  Below N = 1024
// the plan takes radices (4, 5, 3, 2) with TP = N/4, so each thread holds one
// radix-4 butterfly per stage: a single slab is a few hundred line pairs, too
// little work to fill the GPU, and the time of a launch is the length of each
// thread's dependent chain, which the wider group halves against radix 8.
// From N = 1024 on (enough line pairs to fill the GPU) the plan is radices
// (8, 5, 4, 3, 2) with TP = N/8.  That throughput plan (PL = 1) is also
// instantiated below N = 1024: it spends about two thirds of the latency plan's
// instructions per line pair, which pays when many launches share the GPU
// (batched simulations, multi-slab launches).  N is a template parameter, so every stride,
// radix and loop bound is a compile-time constant.  Shared-memory indices are padded by one element
// every eight (pad(i) = i + i/8) so the stride-8 writes of the first stage are
// free of bank conflicts.
#pragma once

#include <type_traits>

#include "ibpm_internal.cuh"

// Resident CTAs per SM that the throughput plan's kernels are compiled for
// (the register budget per thread follows from it).
#ifndef IBPM_WIDE_MIN_BLOCKS
#define IBPM_WIDE_MIN_BLOCKS 1
#endif

namespace ibpm {
namespace dstk {

// Transform plans: 0 = latency (radix 4 below N = 1024), 1 = throughput
// (radix 8).  From N = 1024 on both are the radix-8 plan.
__host__ __device__ constexpr bool ct_fine(int N, int PL = 0) { return N < 1024 && PL == 0; }
__host__ __device__ constexpr int ct_plan(int N, int PL) { return N < 1024 ? PL : 0; }
__host__ __device__ constexpr int ct_radix(int N, int s, int PL = 0) {
    int n = N, idx = 0;
    const bool f = ct_fine(N, PL);
    const int rs[5] = {f ? 4 : 8, 5, f ? 3 : 4, f ? 2 : 3, f ? 8 : 2};
    for (int i = 0; i < 5; ++i) {
        while (n % rs[i] == 0) {
            if (idx == s) return rs[i];
            n /= rs[i];
            ++idx;
        }
    }
    return 1;
}
__host__ __device__ constexpr int ct_nstages(int N, int PL = 0) {
    int n = N, s = 0;
    const bool f = ct_fine(N, PL);
    const int rs[5] = {f ? 4 : 8, 5, f ? 3 : 4, f ? 2 : 3, f ? 8 : 2};
    for (int i = 0; i < 5; ++i)
        while (n % rs[i] == 0) { n /= rs[i]; ++s; }
    return n == 1 ? s : -1;
}
__host__ __device__ constexpr int ct_tp(int N, int PL = 0) {
    int t = (((ct_fine(N, PL) ? N / 4 : N / 8) + 31) / 32) * 32;
    return t < 32 ? 32 : t;
}
__host__ __device__ constexpr int ct_pad(int i) { return i + (i >> 3); }
__host__ __device__ constexpr int ct_buf(int N) { return ct_pad(N) + 8; }  // + scan scratch

// Twiddles of stage S (sub-transform length Ns before it, radix R) are stored
// contiguously as T[(r-1)·Ns + k] = exp(+2πi k r/(Ns R)), r = 1…R-1, k < Ns, so
// the threads of a stage (consecutive k) read consecutive entries.
__host__ __device__ constexpr int ct_stage_ns(int N, int S, int PL = 0) {
    int ns = 1;
    for (int s = 0; s < S; ++s) ns *= ct_radix(N, s, PL);
    return ns;
}
__host__ __device__ constexpr int ct_tw_off(int N, int S, int PL = 0) {
    int off = 0;
    for (int s = 0; s < S; ++s) {
        const int ns = ct_stage_ns(N, s, PL);
        if (ns > 1) off += (ct_radix(N, s, PL) - 1) * ns;
    }
    return off;
}
__host__ __device__ constexpr int ct_tw_count(int N, int PL = 0) { return ct_tw_off(N, ct_nstages(N, PL), PL); }
// Groups (line pairs) per CTA of the x-pass: up to 128 threads, or one group.
__host__ __device__ constexpr int ct_groups(int N, int PL = 0) {
    return ct_tp(N, PL) >= 128 ? 1 : 128 / ct_tp(N, PL);
}

// Complex arithmetic for both precisions (V = double2 or float2).
template <class T> struct cplx_of;
template <> struct cplx_of<double> { using type = double2; };
template <> struct cplx_of<float> { using type = float2; };
template <class T> using cplx_t = typename cplx_of<T>::type;

__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cmuli(double2 a) { return make_double2(-a.y, a.x); }  // i·a
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cmuli(float2 a) { return make_float2(-a.y, a.x); }
template <class V, class T> __device__ __forceinline__ V cmk(T a, T b) { return V{a, b}; }

// Small DFTs with the +2πi sign: V_b = Σ_a v_a e^{+2πi ab/R}.
template <int R, class T> struct dft_t;

template <class T> struct dft_t<2, T> {
    using V = cplx_t<T>;
    __device__ __forceinline__ static void run(V* v) {
        const V t = v[0];
        v[0] = cadd(t, v[1]);
        v[1] = csub(t, v[1]);
    }
};

template <class T> struct dft_t<3, T> {
    using V = cplx_t<T>;
    __device__ __forceinline__ static void run(V* v) {
        const T h3 = T(0.86602540378443864676);  // √3 / 2
        const V s = cadd(v[1], v[2]);
        const V d = csub(v[1], v[2]);
        const V a = V{v[0].x - T(0.5) * s.x, v[0].y - T(0.5) * s.y};
        const V b = V{-h3 * d.y, h3 * d.x};  // i (√3/2) d
        v[0] = cadd(v[0], s);
        v[1] = cadd(a, b);
        v[2] = csub(a, b);
    }
};

template <class T> struct dft_t<4, T> {
    using V = cplx_t<T>;
    __device__ __forceinline__ static void run(V* v) {
        const V t0 = cadd(v[0], v[2]);
        const V t1 = csub(v[0], v[2]);
        const V t2 = cadd(v[1], v[3]);
        const V t3 = cmuli(csub(v[1], v[3]));
        v[0] = cadd(t0, t2);
        v[2] = csub(t0, t2);
        v[1] = cadd(t1, t3);
        v[3] = csub(t1, t3);
    }
};

template <class T> struct dft_t<5, T> {
    using V = cplx_t<T>;
    __device__ __forceinline__ static void run(V* v) {
        const T c1 = T(0.30901699437494742410);   // cos(2π/5)
        const T c2 = T(-0.80901699437494742410);  // cos(4π/5)
        const T s1 = T(0.95105651629515357212);   // sin(2π/5)
        const T s2 = T(0.58778525229247312917);   // sin(4π/5)
        const V s14 = cadd(v[1], v[4]), d14 = csub(v[1], v[4]);
        const V s23 = cadd(v[2], v[3]), d23 = csub(v[2], v[3]);
        const V a1 = V{v[0].x + c1 * s14.x + c2 * s23.x, v[0].y + c1 * s14.y + c2 * s23.y};
        const V a2 = V{v[0].x + c2 * s14.x + c1 * s23.x, v[0].y + c2 * s14.y + c1 * s23.y};
        const V b1 = cmuli(V{s1 * d14.x + s2 * d23.x, s1 * d14.y + s2 * d23.y});
        const V b2 = cmuli(V{s2 * d14.x - s1 * d23.x, s2 * d14.y - s1 * d23.y});
        v[0] = cadd(v[0], cadd(s14, s23));
        v[1] = cadd(a1, b1);
        v[4] = csub(a1, b1);
        v[2] = cadd(a2, b2);
        v[3] = csub(a2, b2);
    }
};

template <class T> struct dft_t<8, T> {
    using V = cplx_t<T>;
    __device__ __forceinline__ static void run(V* v) {
        const T r2 = T(0.70710678118654752440);  // √2 / 2
        V e[4] = {v[0], v[2], v[4], v[6]};
        V o[4] = {v[1], v[3], v[5], v[7]};
        dft_t<4, T>::run(e);
        dft_t<4, T>::run(o);
        o[1] = V{r2 * (o[1].x - o[1].y), r2 * (o[1].x + o[1].y)};    // × e^{iπ/4}
        o[2] = cmuli(o[2]);                                          // × i
        o[3] = V{-r2 * (o[3].x + o[3].y), r2 * (o[3].x - o[3].y)};   // × e^{3iπ/4}
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            v[b] = cadd(e[b], o[b]);
            v[b + 4] = csub(e[b], o[b]);
        }
    }
};

// Synchronise the TP threads of group `gid` of the G groups of a CTA (named
// barrier 1 + gid when the group spans several warps).
// The barrier id is an immediate in each branch, so ptxas reserves only the
// barriers a kernel can use (a run-time id reserves all sixteen, which caps
// the resident blocks per SM).
template <int TP, int G> __device__ __forceinline__ void gsync(int gid) {
    static_assert(G >= 1 && (TP == 32 || G <= 4), "at most four multi-warp groups per CTA");
    if constexpr (TP == 32) {
        __syncwarp();
    } else if constexpr (G == 1) {
        asm volatile("bar.sync 1, %0;" ::"n"(TP) : "memory");
    } else {
        switch (gid) {
            case 0: asm volatile("bar.sync 1, %0;" ::"n"(TP) : "memory"); break;
            case 1: asm volatile("bar.sync 2, %0;" ::"n"(TP) : "memory"); break;
            case 2: asm volatile("bar.sync 3, %0;" ::"n"(TP) : "memory"); break;
            default: asm volatile("bar.sync 4, %0;" ::"n"(TP) : "memory"); break;
        }
    }
}

template <int N, int TP, int G, int R, int Ns, int TWOFF, class T>
__device__ __forceinline__ void fft_stage(cplx_t<T>* buf, const cplx_t<T>* W, int tid, int gid) {
    using V = cplx_t<T>;
    constexpr int nb = N / R;
    constexpr int QM = (nb + TP - 1) / TP;
    constexpr bool exact = (QM * TP == nb);
    V v[QM][R];
#pragma unroll
    for (int q = 0; q < QM; ++q) {
        const int b = tid + q * TP;
        if (exact || b < nb) {
#pragma unroll
            for (int r = 0; r < R; ++r) v[q][r] = buf[ct_pad(b + r * nb)];
        }
    }
    gsync<TP, G>(gid);
#pragma unroll
    for (int q = 0; q < QM; ++q) {
        const int b = tid + q * TP;
        if (exact || b < nb) {
            const int k = b % Ns;
            if constexpr (Ns > 1) {
#pragma unroll
                for (int r = 1; r < R; ++r) v[q][r] = cmul(v[q][r], W[TWOFF + (r - 1) * Ns + k]);
            }
            dft_t<R, T>::run(v[q]);
            const int base = (b - k) * R + k;
#pragma unroll
            for (int r = 0; r < R; ++r) buf[ct_pad(base + r * Ns)] = v[q][r];
        }
    }
    gsync<TP, G>(gid);
}

template <int N, int TP, int G, int S, int Ns, class T, int PL>
__device__ __forceinline__ void fft_stages(cplx_t<T>* buf, const cplx_t<T>* W, int tid, int gid) {
    if constexpr (S < ct_nstages(N, PL)) {
        constexpr int R = ct_radix(N, S, PL);
        fft_stage<N, TP, G, R, Ns, ct_tw_off(N, S, PL), T>(buf, W, tid, gid);
        fft_stages<N, TP, G, S + 1, Ns * R, T, PL>(buf, W, tid, gid);
    }
}

// Pre-processing: buf[m] = y_m from load(m-1) = (a_{m-1}, b_{m-1}).
template <int N, int TP, class T, class Load>
__device__ __forceinline__ void dst_pre(cplx_t<T>* buf, const T* s, int tid, Load load) {
    using V = cplx_t<T>;
    constexpr int half = N >> 1;
    constexpr int IT = (half + TP) / TP;  // m = tid + it·TP covers 0 … half
    V fm[IT], fn[IT];
#pragma unroll
    for (int it = 0; it < IT; ++it) {  // issue every load before using any
        const int m = tid + it * TP;
        if (m >= 1 && m <= half) {
            fm[it] = load(m - 1);
            if (m < half) fn[it] = load(N - m - 1);
        }
    }
#pragma unroll
    for (int it = 0; it < IT; ++it) {
        const int m = tid + it * TP;
        if (m == 0) {
            buf[0] = V{T(0), T(0)};
        } else if (m == half) {  // sin(π/2) = 1
            buf[ct_pad(m)] = V{T(2) * fm[it].x, T(2) * fm[it].y};
        } else if (m < half) {
            const T sm = s[m];
            const V sum = cadd(fm[it], fn[it]), dif = csub(fm[it], fn[it]);
            const V ys = V{sm * sum.x, sm * sum.y};
            buf[ct_pad(m)] = V{ys.x + T(0.5) * dif.x, ys.y + T(0.5) * dif.y};
            buf[ct_pad(N - m)] = V{ys.x - T(0.5) * dif.x, ys.y - T(0.5) * dif.y};
        }
    }
}

__device__ __forceinline__ double2 shfl_up2(double2 v, int off) {
    return make_double2(__shfl_up_sync(0xffffffffu, v.x, off), __shfl_up_sync(0xffffffffu, v.y, off));
}
__device__ __forceinline__ float2 shfl_up2(float2 v, int off) {
    return make_float2(__shfl_up_sync(0xffffffffu, v.x, off), __shfl_up_sync(0xffffffffu, v.y, off));
}

// Exclusive prefix sum of one complex value per thread over the TP threads of
// a group.
template <int TP, int G, class V>
__device__ __forceinline__ V group_excl_scan(V v, int tid, int gid, V* scratch) {
    const int lane = tid & 31, w = tid >> 5;
    V inc = v;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const V n = shfl_up2(inc, off);
        if (lane >= off) inc = cadd(inc, n);
    }
    V ex = shfl_up2(inc, 1);
    if (lane == 0) ex = V{0, 0};
    if constexpr (TP > 32) {
        if (lane == 31) scratch[w] = inc;
        gsync<TP, G>(gid);
        V base = V{0, 0};
        for (int u = 0; u < w; ++u) base = cadd(base, scratch[u]);
        ex = cadd(base, ex);
    }
    return ex;
}

// Post-processing: from Z (in buf) produce the N-1 outputs of both lines and
// hand them to emit(o, (a_o, b_o)).  All reads of buf precede every emit, so
// emit may write into buf.
template <int N, int TP, int G, class T, class Emit>
__device__ __forceinline__ void dst_post(cplx_t<T>* buf, int tid, int gid, cplx_t<T>* scratch, Emit emit) {
    using V = cplx_t<T>;
    constexpr int half = N >> 1;
    constexpr int C = (half + TP - 1) / TP;
    const int k0 = tid * C;
    V D[C], O[C];
    V tot = V{T(0), T(0)};
#pragma unroll
    for (int t = 0; t < C; ++t) {
        const int k = k0 + t;
        if (k < half) {
            const V zk = buf[ct_pad(k)];
            V d;
            if (k == 0) {
                d = zk;
                O[t] = V{T(0), T(0)};
            } else {
                const V zn = buf[ct_pad(N - k)];
                d = cadd(zk, zn);
                const V dl = csub(zk, zn);
                O[t] = V{dl.y, -dl.x};  // −i (Z_k − Z_{N−k})
            }
            tot = cadd(tot, d);
            D[t] = tot;
        }
    }
    const V ex = group_excl_scan<TP, G>(tot, tid, gid, scratch);
    gsync<TP, G>(gid);
#pragma unroll
    for (int t = 0; t < C; ++t) {
        const int k = k0 + t;
        if (k < half) {
            emit(2 * k, cadd(ex, D[t]));
            if (k > 0) emit(2 * k - 1, O[t]);
        }
    }
}

// One DST-I of a line pair: load → pre → FFT (plan PL) → post → emit.
template <int N, int TP, int G, class T, int PL = 0, class Load, class Emit>
__device__ __forceinline__ void dst_pair(cplx_t<T>* buf, const cplx_t<T>* W, const T* s, int tid, int gid,
                                         Load load, Emit emit) {
    dst_pre<N, TP, T>(buf, s, tid, load);
    gsync<TP, G>(gid);
    fft_stages<N, TP, G, 0, 1, T, PL>(buf, W, tid, gid);
    dst_post<N, TP, G, T>(buf, tid, gid, buf + ct_pad(N), emit);
}

// Tables of one precision: stage twiddles, sin(π m/N) and the spectral table
// used by the divide (FP64: cos(π(k+1)/N); FP32: 4 sin²(π(k+1)/(2N))).
template <class T> struct Tabs {
    const cplx_t<T>* W;
    const T* s;
    const T* c;
};
// The stage twiddles are those of plan PL (W / W32: latency plan, Wt / Wt32:
// throughput plan).
template <class T> __host__ __device__ Tabs<T> tabs_of(const DstPlan& p, int PL = 0);
template <> __host__ __device__ inline Tabs<double> tabs_of<double>(const DstPlan& p, int PL) {
    return {PL ? p.Wt : p.W, p.s, p.c};
}
template <> __host__ __device__ inline Tabs<float> tabs_of<float>(const DstPlan& p, int PL) {
    return {PL ? p.Wt32 : p.W32, p.s32, p.a32};
}

// Copy the transform tables into shared memory: stage twiddles (complex),
// then sin(πm/N) for m ≤ N/2.
template <int N, class T, int PL = 0>
__device__ __forceinline__ void stage_tables(cplx_t<T>* tw, T* sn, const Tabs<T>& p) {
    for (int i = threadIdx.x; i < ct_tw_count(N, PL); i += blockDim.x) cp_async<sizeof(cplx_t<T>)>(tw + i, p.W + i);
    for (int i = threadIdx.x; i <= N / 2; i += blockDim.x) cp_async<sizeof(T)>(sn + i, p.s + i);
}
template <int N, class T, int PL = 0>
__host__ __device__ constexpr size_t tables_bytes() {
    return (size_t)ct_tw_count(N, PL) * sizeof(cplx_t<T>) + (size_t)((N / 2 + 4) & ~3) * sizeof(T);
}

// ---------------------------------------------------------------------------
// x-pass: lines are rows of a slab (contiguous).  One group per line pair.
// ---------------------------------------------------------------------------
template <int LOAD>
using x_real_t = std::conditional_t<(LOAD == XLOAD_PLAIN || LOAD == XLOAD_BC || LOAD == XLOAD_SUM), double, float>;
template <int LOAD>
__host__ __device__ constexpr bool x_res() { return LOAD == XLOAD_RES_LAP || LOAD == XLOAD_RES_A; }
// Shared memory of the x-pass: tables, one FFT buffer per group, and for the
// residual loads six staged rows of N doubles per group (16-byte aligned).
template <int N, int LOAD, int PL>
__host__ __device__ constexpr size_t x_res_off() {
    return ((tables_bytes<N, x_real_t<LOAD>, PL>() +
             (size_t)ct_groups(N, PL) * ct_buf(N) * sizeof(cplx_t<x_real_t<LOAD>>) + 15) / 16) * 16;
}
template <int N, int LOAD, int PL>
__host__ __device__ constexpr size_t x_smem_bytes() {
    return x_res_off<N, LOAD, PL>() + (x_res<LOAD>() ? (size_t)ct_groups(N, PL) * 6 * N * sizeof(double) : 0);
}

template <int N, int LOAD, int EMIT, int PL>
__global__ void __launch_bounds__(ct_groups(N, PL) * ct_tp(N, PL), ct_fine(N, PL) ? 1 : IBPM_WIDE_MIN_BLOCKS)
    dst_x_kernel(XPassArgs a, Geom g, DstPlan p) {
    using T = x_real_t<LOAD>;
    using V = cplx_t<T>;
    constexpr int TP = ct_tp(N, PL);
    constexpr int G = ct_groups(N, PL);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V* tw = reinterpret_cast<V*>(smem_raw);
    T* sn = reinterpret_cast<T*>(tw + ct_tw_count(N, PL));
    V* bufs = reinterpret_cast<V*>(smem_raw + tables_bytes<N, T, PL>());
    stage_tables<N, T, PL>(tw, sn, tabs_of<T>(p, PL));  // constant tables: before the dependency wait
    cp_async_wait();
    __syncthreads();
    pdl_wait();
    pdl_trigger();
    const int gid = threadIdx.x / TP, tid = threadIdx.x % TP;
    V* buf = bufs + gid * ct_buf(N);
    constexpr bool RES = x_res<LOAD>();
    const int la = a.line0 + 2 * (blockIdx.x * G + gid);
    if (la >= a.line1) return;  // the whole group leaves together
    const bool hasb = (la + 1) < a.line1;
    const int y = blockIdx.y;
    const int P = g.P, n1 = g.n1, n2 = g.n2;
    const long long ioff = a.in_map.off(y) + (long long)la * P;

    CoarseBC cb;
    cb.rc = nullptr; cb.P = P; cb.nx = g.nx; cb.ny = g.ny;
    if ((LOAD == XLOAD_BC || LOAD == XLOAD_RES_LAP) && a.coarse && a.in_map.level(y) + 1 < g.mg)
        cb.rc = a.coarse + a.coarse_map.off(y);
    const double* xg = (LOAD == XLOAD_RES_LAP || LOAD == XLOAD_RES_A) ? a.aux + a.aux_map.off(y) : nullptr;
    const double cA = (LOAD == XLOAD_RES_A && a.mcA) ? a.mcA[a.in_map.batch(y)] : a.cA;

    // apply_bc!(r, get_bc!(coarse), 1.0) (mg-utils.jl:43-60) in the reference's
    // order: bottom row, top row, left column, right column.
    auto with_bc = [&](double v, int i, int j) -> double {
        if (j == 0) v += cb.bot(i + 1);
        if (j == n2 - 1) v += cb.top(i + 1);
        if (i == 0) v += cb.left(j + 1);
        if (i == n1 - 1) v += cb.right(j + 1);
        return v;
    };
    // Residual loads: the group stages x̃ rows la-1 … la+2 (zero outside the
    // slab) and b rows la, la+1 in shared memory, rows of stride N doubles.
    double* rs = RES ? reinterpret_cast<double*>(smem_raw + x_res_off<N, LOAD, PL>()) + (size_t)gid * 6 * N : nullptr;
    if constexpr (RES) {
        const double* bin = static_cast<const double*>(a.in) + a.in_map.off(y);
#pragma unroll 1
        for (int r = 0; r < 6; ++r) {
            const int j = r < 4 ? la - 1 + r : la + r - 4;
            const bool valid = j >= 0 && j < n2 && (r != 5 || hasb);
            const double* src = (r < 4 ? xg : bin) + (long long)j * P;
            double* dst = rs + r * N;
            for (int i = 2 * tid; i < n1; i += 2 * TP) {
                if (valid) {
                    if (i + 1 < n1) cp_async16(dst + i, src + i);
                    else cp_async8(dst + i, src + i);
                } else {
                    dst[i] = 0.0;
                    if (i + 1 < n1) dst[i + 1] = 0.0;
                }
            }
        }
        cp_async_wait();
        gsync<TP, G>(gid);
    }
    // L x̃ at (i, la + r) = 4 x̃ − Σ neighbours, zero beyond the slab edges
    // (r = 0, 1; staged row 1 + r)
    auto lap = [&](int i, int r) -> double {
        const double* c = rs + (1 + r) * N + i;
        double nb = 0.0;
        if (i > 0) nb += c[-1];
        if (i + 1 < n1) nb += c[1];
        nb += c[-N];
        nb += c[N];
        return 4.0 * c[0] - nb;
    };
    auto line_val = [&](const double* row, int i, int j) -> double {
        double v = row[i];
        if constexpr (LOAD == XLOAD_BC) {
            if (cb.rc) v = with_bc(v, i, j);
        }
        return v;
    };
    auto res_val = [&](int i, int r) -> double {
        double v = rs[(4 + r) * N + i];
        if constexpr (LOAD == XLOAD_RES_LAP) {
            if (cb.rc) v = with_bc(v, i, la + r);
            v -= lap(i, r);
        } else {
            v -= rs[(1 + r) * N + i] + cA * lap(i, r);
        }
        return v;
    };
    auto load = [&](int i) -> V {
        if constexpr (LOAD == XLOAD_F32) {
            const float* ra = static_cast<const float*>(a.in) + ioff;
            return V{ra[i], hasb ? ra[i + P] : 0.0f};
        } else if constexpr (LOAD == XLOAD_SUM || LOAD == XLOAD_F32_SUM) {
            const T* ra = static_cast<const T*>(a.in) + ioff;
            const T* rb = static_cast<const T*>(a.in2) + a.in2_map.off(y) + (long long)la * P;
            return V{ra[i] + rb[i], hasb ? ra[i + P] + rb[i + P] : T(0)};
        } else if constexpr (RES) {
            return V{(T)res_val(i, 0), hasb ? (T)res_val(i, 1) : T(0)};
        } else {
            const double* ra = static_cast<const double*>(a.in) + ioff;
            const double va = line_val(ra, i, la);
            const double vb = hasb ? line_val(ra + P, i, la + 1) : 0.0;
            return V{(T)va, (T)vb};
        }
    };
    // Stores that read what they update: fetch those values before the
    // transform, so their latency overlaps it (each thread owns the same
    // columns o = tid + k·TP of both lines throughout).
    constexpr int EO = (N - 1 + TP - 1) / TP;
    constexpr bool READ_OUT = (EMIT == XEMIT_SUB || EMIT == XEMIT_ADD || EMIT == XEMIT_ADD_STORE ||
                               EMIT == XEMIT_ACC_SUB);
    constexpr bool READ_AUX = (EMIT == XEMIT_ADD_FROM || EMIT == XEMIT_ACC_SUB);
    const long long ooff = a.out_map.off(y) + (long long)la * P;
    double po[EO][2], px[EO][2];
    if constexpr (READ_OUT || READ_AUX) {
        const double* oa = static_cast<const double*>(a.out) + ooff;
        const double* xa = READ_AUX ? a.aux + a.aux_map.off(y) + (long long)la * P : nullptr;
#pragma unroll
        for (int k = 0; k < EO; ++k) {
            const int o = tid + k * TP;
            if (o < n1) {
                if constexpr (READ_OUT) {
                    po[k][0] = oa[o];
                    po[k][1] = hasb ? oa[o + P] : 0.0;
                }
                if constexpr (READ_AUX) {
                    px[k][0] = xa[o];
                    px[k][1] = hasb ? xa[o + P] : 0.0;
                }
            }
        }
    }
    dst_pair<N, TP, G, T, PL>(buf, tw, sn, tid, gid, load, [&](int o, V v) { buf[ct_pad(o)] = v; });
    gsync<TP, G>(gid);
#pragma unroll
    for (int k = 0; k < EO; ++k) {
        const int o = tid + k * TP;
        if (o >= n1) break;
        const V v = buf[ct_pad(o)];
        if constexpr (EMIT == XEMIT_F32) {
            float* oa = static_cast<float*>(a.out) + ooff;
            oa[o] = (float)v.x;
            if (hasb) oa[o + P] = (float)v.y;
        } else {
            double* oa = static_cast<double*>(a.out) + ooff;
            if constexpr (EMIT == XEMIT_STORE) {
                oa[o] = v.x;
                if (hasb) oa[o + P] = v.y;
            } else if constexpr (EMIT == XEMIT_SUB) {
                oa[o] = po[k][0] - v.x;
                if (hasb) oa[o + P] = po[k][1] - v.y;
            } else if constexpr (EMIT == XEMIT_ADD) {
                oa[o] = po[k][0] + (double)v.x;
                if (hasb) oa[o + P] = po[k][1] + (double)v.y;
            } else if constexpr (EMIT == XEMIT_ADD_FROM) {
                oa[o] = px[k][0] + (double)v.x;
                if (hasb) oa[o + P] = px[k][1] + (double)v.y;
            } else if constexpr (EMIT == XEMIT_ADD_STORE) {
                double* xa = a.aux + a.aux_map.off(y) + (long long)la * P;
                oa[o] = po[k][0] + v.x;
                xa[o] = v.x;
                if (hasb) {
                    oa[o + P] = po[k][1] + v.y;
                    xa[o + P] = v.y;
                }
            } else {  // XEMIT_ACC_SUB
                double* xa = a.aux + a.aux_map.off(y) + (long long)la * P;
                const double pa = px[k][0] + (double)v.x;
                xa[o] = pa;
                oa[o] = po[k][0] - pa;
                if (hasb) {
                    const double pb = px[k][1] + (double)v.y;
                    xa[o + P] = pb;
                    oa[o + P] = po[k][1] - pb;
                }
            }
        }
    }
}

// ---------------------------------------------------------------------------
// y-pass of a Poisson-type solve on a tile of TW = 2G columns (all rows)
// staged in shared memory, in place: DST-I, spectral divide, DST-I.
// ---------------------------------------------------------------------------
// Groups (column pairs) per CTA of the y-pass.  FP32 passes take one group
// (more CTAs for a single slab: the refined step's y-passes are single-slab
// and latency-bound); FP64 passes keep at least two with the fine plan, so a
// CTA reads tiles of four 8-byte columns.
template <int N, class T, int PL>
__host__ __device__ constexpr int y_groups() {
    return (std::is_same<T, double>::value && ct_fine(N, PL) && ct_groups(N, PL) < 2) ? 2 : ct_groups(N, PL);
}
template <int N, class T, int PL>
__host__ __device__ constexpr int y_threads() { return y_groups<N, T, PL>() * ct_tp(N, PL); }
template <int N, class T, int PL>
__host__ __device__ constexpr int y_tile_w() { return 2 * y_groups<N, T, PL>(); }
__host__ __device__ constexpr int round4(int n) { return ((n + 3) / 4) * 4; }
// The column tile is column-major, element (row j, column c) at
// c·CS + j + ⌊j/PI⌋: one pad element every PI rows.  E is the number of
// elements in one 128-byte line, the period of the shared-memory banks.
// Each thread of the post-processing scan owns a run of C consecutive
// outputs, so one warp access writes rows 2C apart.  PI = E·(odd part of C)
// puts those 32 rows into distinct banks, except where they wrap past two
// pads (for C = 1, 2, 4 a pad every line; for C = 3, one every three lines),
// and consecutive rows (the transform's reads, the divide) meet at most one
// pad per access.  CS ≡ E/TW (mod E)
// makes the row-major fill and store (TW columns of E/TW rows per access)
// conflict-free too.
template <class T>
__host__ __device__ constexpr int y_line_elems() { return 128 / (int)sizeof(T); }
template <int N, int PL>
__host__ __device__ constexpr int y_scan_run() { return (N / 2 + ct_tp(N, PL) - 1) / ct_tp(N, PL); }
template <int N, class T, int PL>
__host__ __device__ constexpr int y_pad_every() {
    int c = y_scan_run<N, PL>();
    while (c % 2 == 0) c /= 2;
    return y_line_elems<T>() * c;
}
template <int N, class T, int PL>
__host__ __device__ constexpr int y_off(int j) { return j + j / y_pad_every<N, T, PL>(); }
template <int N, class T, int PL>
__host__ __device__ constexpr int y_col_stride(int n2) {
    constexpr int E = y_line_elems<T>();
    constexpr int TW = 2 * y_groups<N, T, PL>();
    constexpr int R = (E / TW) > 0 ? E / TW : 1;
    const int base = y_off<N, T, PL>(n2 - 1) + 2;   // one spare element past the last row
    return base + ((R - base % E) % E + E) % E;
}
template <int N, class T, int PL>
__host__ __device__ constexpr int y_tile_elems(int n2) {
    return round4(2 * y_groups<N, T, PL>() * y_col_stride<N, T, PL>(n2));
}
// Scratch of the edge-source synthesis (SYNTH): per-warp partial sums of the
// bottom and top rows' sine transforms, then the sums themselves.
template <int N, class T, int PL>
__host__ __device__ constexpr int y_synth_slots() {
    return (y_threads<N, T, PL>() / 32 + 2) * 2 * y_tile_w<N, T, PL>();
}
template <int N, class T, int PL, bool SYNTH = false>
__host__ __device__ constexpr size_t y_smem_bytes(int n2) {
    return tables_bytes<N, T, PL>() + (size_t)round4(n2) * sizeof(T) +  // spectral table of y
           (size_t)y_tile_elems<N, T, PL>(n2) * sizeof(T) +
           (size_t)y_groups<N, T, PL>() * ct_buf(N) * sizeof(cplx_t<T>) +
           (SYNTH ? (size_t)y_synth_slots<N, T, PL>() * sizeof(double) : 0);
}

// SYNTH: the input is not read but built, the x-spectrum of apply_bc!(e_ℓ)
// for the edge vector of the slab's level (BtSynth): with S(i, k) =
// 2 sin(π i k / nx) the x-pass's sine transform,
//     X(k, j) = S(1, k) e_L(j) + S(nx−1, k) e_R(j)
//             + [j = 1] Σ_i S(i, k) e_B(i) + [j = ny−1] Σ_i S(i, k) e_T(i),
// and the result goes to `out` (same slab map) instead of back into `data`.
template <int N, class T, int PL, bool SYNTH = false>
// (3 resident 256-thread CTAs per SM keep the FP64 pass at 80 registers without
// spills: the five-slab trial solve's y-pass then needs 1.4 waves instead of 2.2)
__global__ void __launch_bounds__(y_threads<N, T, PL>(),
                                  N > 512 ? 1 : (!ct_fine(N, PL) ? IBPM_WIDE_MIN_BLOCKS
                                                                 : (y_threads<N, T, PL>() <= 128 ? 5 : 3)))
    dst_y_kernel(T* data, SlabMap map, Geom g, DstPlan p, const T* __restrict__ cx, SpecParams sp,
                 T* out = nullptr, BtSynth bs = BtSynth{}) {
    using V = cplx_t<T>;
    constexpr int TP = ct_tp(N, PL);
    constexpr int G = y_groups<N, T, PL>();
    constexpr int TW = y_tile_w<N, T, PL>();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int P = g.P, n1 = g.n1, n2 = g.n2;
    const Tabs<T> tb = tabs_of<T>(p, PL);
    V* tw = reinterpret_cast<V*>(smem_raw);
    T* sn = reinterpret_cast<T*>(tw + ct_tw_count(N, PL));
    T* cyv = reinterpret_cast<T*>(smem_raw + tables_bytes<N, T, PL>());
    T* tile = cyv + round4(n2);
    const int tile_d = y_tile_elems<N, T, PL>(n2);
    constexpr int CS = y_col_stride<N, T, PL>(N - 1);   // n2 = N − 1 in the y-pass
    auto off = [](int j) -> int { return y_off<N, T, PL>(j); };   // row j within a column
    auto at = [&](int j, int c) -> int { return c * CS + off(j); };
    const int gid = threadIdx.x / TP, tid = threadIdx.x % TP;
    V* buf = reinterpret_cast<V*>(tile + tile_d) + gid * ct_buf(N);
    const int i0 = blockIdx.x * TW;
    T* base = data + map.off(blockIdx.y);
    const int lev = map.level(blockIdx.y);

    stage_tables<N, T, PL>(tw, sn, tb);  // constant tables: before the dependency wait
    for (int j = threadIdx.x; j < n2; j += blockDim.x) cp_async<sizeof(T)>(cyv + j, tb.c + j);
    pdl_wait();
    pdl_trigger();
    if constexpr (SYNTH) {
        // the edge vectors and the sums over them are FP64 (they couple the
        // levels); the tile takes the x-spectrum rounded to T
        const int ep = ((2 * n1 + 2 * n2) + 3) & ~3;
        const double* e = static_cast<const double*>(bs.e) + ((long long)map.batch(blockIdx.y) * g.mg + lev) * ep;
        const double* sxt = static_cast<const double*>(bs.sx);
        const int nx = bs.nx, nx2 = 2 * bs.nx;
        auto sinpix = [&](int t) -> double {  // sin(π t / nx), 0 ≤ t < 2 nx
            return t < nx ? __ldg(&sxt[t]) : -__ldg(&sxt[t - nx]);
        };
        double* red = reinterpret_cast<double*>(reinterpret_cast<unsigned char*>(tile + tile_d) +
                                                (size_t)G * ct_buf(N) * sizeof(V));
        // bottom and top rows: Σ_i S(i, k) e(i) for the CTA's columns k, the
        // sine argument (i + 1) k mod 2nx advanced by a fixed step per thread
        double accB[TW], accT[TW];
        int tk[TW], dk[TW];
#pragma unroll
        for (int c = 0; c < TW; ++c) {
            accB[c] = accT[c] = 0.0;
            const int k = i0 + c + 1;
            tk[c] = (int)(((long long)(threadIdx.x + 1) * k) % nx2);
            dk[c] = (int)(((long long)blockDim.x * k) % nx2);
        }
#pragma unroll 4
        for (int i = threadIdx.x; i < n1; i += blockDim.x) {
            const double eb = __ldg(&e[i]), et = __ldg(&e[n1 + i]);
#pragma unroll
            for (int c = 0; c < TW; ++c) {
                const double sv = 2.0 * sinpix(tk[c]);
                accB[c] += sv * eb;
                accT[c] += sv * et;
                tk[c] += dk[c];
                if (tk[c] >= nx2) tk[c] -= nx2;
            }
        }
        const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
        for (int c = 0; c < TW; ++c) {
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) {
                accB[c] += __shfl_xor_sync(0xffffffffu, accB[c], off);
                accT[c] += __shfl_xor_sync(0xffffffffu, accT[c], off);
            }
            if (lane == 0) {
                red[w * 2 * TW + c] = accB[c];
                red[w * 2 * TW + TW + c] = accT[c];
            }
        }
        __syncthreads();
        if (threadIdx.x < 2 * TW) {
            double acc = 0.0;
            for (int u = 0; u < nw; ++u) acc += red[u * 2 * TW + threadIdx.x];
            red[nw * 2 * TW + threadIdx.x] = acc;
        } else if (threadIdx.x < 4 * TW) {
            // S(1, k) and S(nx − 1, k) of the column c
            const int c = (threadIdx.x - 2 * TW) >> 1;
            const long long k = i0 + c + 1;
            const int t = (int)(((threadIdx.x & 1) ? k * (nx - 1) : k) % nx2);
            red[(nw + 1) * 2 * TW + (threadIdx.x - 2 * TW)] = 2.0 * sinpix(t);
        }
        __syncthreads();
        const double* bh = red + nw * 2 * TW;         // [0, TW): bottom, [TW, 2TW): top
        const double* sLR = red + (nw + 1) * 2 * TW;  // [2c]: S(1, k_c), [2c + 1]: S(nx−1, k_c)
        const double* eL = e + 2 * n1;
        const double* eR = eL + n2;
        // (the loads of eight steps in flight: the loop is a chain of L2 reads otherwise)
#pragma unroll 8
        for (int idx = threadIdx.x; idx < n2 * TW; idx += blockDim.x) {
            const int j = idx / TW, c = idx - j * TW;
            const int i = i0 + c;
            double v = 0.0;
            if (i < n1) {
                v = sLR[2 * c] * __ldg(&eL[j]) + sLR[2 * c + 1] * __ldg(&eR[j]);
                if (j == 0) v += bh[c];
                if (j == n2 - 1) v += bh[TW + c];
            }
            tile[at(j, c)] = (T)v;
        }
        __syncthreads();
    } else {
        for (int idx = threadIdx.x; idx < n2 * TW; idx += blockDim.x) {
            const int j = idx / TW, c = idx - j * TW;
            const int i = i0 + c;
            if (i < n1) cp_async<sizeof(T)>(tile + at(j, c), base + (long long)j * P + i);
            else tile[at(j, c)] = T(0);
        }
        cp_async_wait();
        __syncthreads();
    }

    const int ca = 2 * gid;
    const int ia = i0 + ca;
    if (ia < n1) {
        const bool hasb = ia + 1 < n1;
        T* const colA = tile + ca * CS;   // the group's two columns
        T* const colB = colA + CS;
        auto load = [&](int m) -> V { return V{colA[off(m)], colB[off(m)]}; };
        auto emit = [&](int o, V v) {
            colA[off(o)] = v.x;
            colB[off(o)] = v.y;
        };
        auto divide = [&]() {
            if constexpr (std::is_same<T, double>::value) {
                // w ./= M ; w .*= scale  with Λ = -2 (cos(π i/nx) + cos(π j/ny) - 2)
                // (laplacian.jl:17-41, 61-71)
                const double cxa = __ldg(&cx[ia]);
                const double cxb = hasb ? __ldg(&cx[ia + 1]) : 0.0;
                const double* md = sp.mden ? sp.mden + (long long)map.batch(blockIdx.y) * 9 : nullptr;
                const double den = md ? md[lev] : sp.den[lev];
                const double dt = md ? md[8] : sp.dt;
                for (int o = tid; o < n2; o += TP) {
                    const double c2 = cyv[o];
                    const double la = -2.0 * ((cxa + c2) - 2.0);
                    const double lb = -2.0 * ((cxb + c2) - 2.0);
                    double Ma, Mb;
                    if (sp.mode == SPEC_DELTA) {
                        Ma = la;
                        Mb = lb;
                    } else {
                        Ma = 1.0 + la * dt / den;
                        Mb = 1.0 + lb * dt / den;
                    }
                    const int oo = off(o);
                    colA[oo] = (colA[oo] * nr_rcp(Ma)) * sp.scale;
                    colB[oo] = hasb ? (colB[oo] * nr_rcp(Mb)) * sp.scale : 0.0;
                }
            } else {
                // the same divisor from Λ = a_x(i) + a_y(j), a(k) = 4 sin²(πk/(2n)):
                // no cancellation for the smallest eigenvalues in FP32
                const float axa = __ldg(&cx[ia]);
                const float axb = hasb ? __ldg(&cx[ia + 1]) : 0.0f;
                const double* md = sp.mden ? sp.mden + (long long)map.batch(blockIdx.y) * 9 : nullptr;
                const float kf = (sp.mode == SPEC_DELTA) ? 0.0f
                                 : md ? (float)(md[8] / md[lev]) : (float)(sp.dt / sp.den[lev]);
                const float sc = (float)sp.scale;
                for (int o = tid; o < n2; o += TP) {
                    const float la = axa + cyv[o];
                    const float lb = axb + cyv[o];
                    const float Ma = (sp.mode == SPEC_DELTA) ? la : fmaf(la, kf, 1.0f);
                    const float Mb = (sp.mode == SPEC_DELTA) ? lb : fmaf(lb, kf, 1.0f);
                    const int oo = off(o);
                    colA[oo] = colA[oo] * (__frcp_rn(Ma) * sc);
                    colB[oo] = hasb ? colB[oo] * (__frcp_rn(Mb) * sc) : 0.0f;
                }
            }
        };
        dst_pair<N, TP, G, T, PL>(buf, tw, sn, tid, gid, load, emit);
        gsync<TP, G>(gid);
        divide();
        gsync<TP, G>(gid);
        dst_pair<N, TP, G, T, PL>(buf, tw, sn, tid, gid, load, emit);
    }
    __syncthreads();
    T* dst = SYNTH ? out + map.off(blockIdx.y) : base;
    for (int idx = threadIdx.x; idx < n2 * TW; idx += blockDim.x) {
        const int j = idx / TW, c = idx - j * TW;
        const int i = i0 + c;
        if (i < n1) dst[(long long)j * P + i] = tile[at(j, c)];
    }
}

// ---------------------------------------------------------------------------
// Line samples of a boundary-transfer vort2flux! (ibpm_internal.cuh, BtSynth)
// from the y-pass output Y (x-spectral, y-physical) of the levels of `map`:
// block 0 of a slab transforms the rows at ny/4 and at 3ny/4 back along x (one
// line pair) and keeps x = nx/4 … 3nx/4; the other blocks form the columns at
// nx/4 and 3nx/4, ψ(i0, j) = Σ_k S(i0, k) Y(k, j), one warp per row j.  There
// S(nx/4, k) = 2 sin(πk/4) and S(3nx/4, k) = 2 sin(3πk/4) repeat with period
// 8 in k.
// ---------------------------------------------------------------------------
template <int N, int PL>
__host__ __device__ constexpr size_t lines_smem_bytes() {
    return tables_bytes<N, double, PL>() + (size_t)ct_buf(N) * sizeof(double2);
}

// T: the type of Y (the FP32 corrections of the refined path or FP64); the
// samples are formed in FP64 either way (they couple the levels).
template <int N, class T, int PL>
__global__ void __launch_bounds__(ct_tp(N, PL)) dst_lines_kernel(const T* Y, SlabMap map, Geom g, DstPlan p,
                                                                 double* samples) {
    using V = double2;
    constexpr int TP = ct_tp(N, PL);
    const int P = g.P, nx = g.nx, ny = g.ny, n1 = g.n1;
    const T* base = Y + map.off(blockIdx.y);
    double* smp = samples + ((long long)map.batch(blockIdx.y) * g.mg + map.level(blockIdx.y)) * (nx + ny + 4);
    if (blockIdx.x == 0) {
        extern __shared__ __align__(16) unsigned char smem_raw[];
        V* tw = reinterpret_cast<V*>(smem_raw);
        double* sn = reinterpret_cast<double*>(tw + ct_tw_count(N, PL));
        V* buf = reinterpret_cast<V*>(smem_raw + tables_bytes<N, double, PL>());
        stage_tables<N, double, PL>(tw, sn, tabs_of<double>(p, PL));
        cp_async_wait();
        __syncthreads();
        pdl_wait();
        pdl_trigger();
        const T* ra = base + (long long)(ny / 4 - 1) * P;
        const T* rb = base + (long long)(3 * ny / 4 - 1) * P;
        const int o0 = nx / 4 - 1, o1 = 3 * nx / 4 - 1;
        double* rowB = smp;
        double* rowT = smp + nx / 2 + 1;
        dst_pair<N, TP, 1, double, PL>(buf, tw, sn, threadIdx.x, 0,
                                       [&](int i) -> V { return V{(double)ra[i], (double)rb[i]}; },
                                       [&](int o, V v) {
                                           if (o >= o0 && o <= o1) {
                                               rowB[o - o0] = v.x;
                                               rowT[o - o0] = v.y;
                                           }
                                       });
        return;
    }
    pdl_wait();
    pdl_trigger();
    const int lane = threadIdx.x & 31;
    const int r = (blockIdx.x - 1) * (TP / 32) + (threadIdx.x >> 5);
    if (r > ny / 2) return;
    const T* row = base + (long long)(ny / 4 - 1 + r) * P;
    const double s2 = 1.41421356237309504880;  // 2 sin(π/4)
    const double wl[8] = {0.0, s2, 2.0, s2, 0.0, -s2, -2.0, -s2};
    const double wr[8] = {0.0, s2, -2.0, s2, 0.0, -s2, 2.0, -s2};
    double aL = 0.0, aR = 0.0;
    for (int m = lane; m < n1; m += 32) {
        const double v = (double)row[m];
        const int k = (m + 1) & 7;
        aL += wl[k] * v;
        aR += wr[k] * v;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        aL += __shfl_xor_sync(0xffffffffu, aL, off);
        aR += __shfl_xor_sync(0xffffffffu, aR, off);
    }
    if (lane == 0) {
        smp[nx + 2 + r] = aL;
        smp[nx + 2 + ny / 2 + 1 + r] = aR;
    }
}

// ---------------------------------------------------------------------------
// Launchers for one compile-time length.
// ---------------------------------------------------------------------------
template <int N, int LOAD, int EMIT, int PL>
cudaError_t launch_x_n(const Geom& g, const DstPlan& px, const XPassArgs& a, cudaStream_t st) {
    constexpr int TP = ct_tp(N, PL);
    constexpr int G = ct_groups(N, PL);
    const int lines = a.line1 - a.line0;
    if (lines <= 0 || a.nslabs <= 0) return cudaSuccess;
    const int pairs = (lines + 1) / 2;
    dim3 grid((pairs + G - 1) / G, a.nslabs);
    const size_t smem = x_smem_bytes<N, LOAD, PL>();
    return launch_k(dst_x_kernel<N, LOAD, EMIT, PL>, grid, dim3(G * TP), smem, st, a, g, px);
}

// The plan of a launch: the plan's single-slab or multi-slab choice; the
// throughput plan needs its twiddle table.
inline int launch_plan(int N, const DstPlan& p, int nslabs) {
    if (p.sims > 1) nslabs /= p.sims;
    int pl = nslabs > 1 ? p.planN : p.plan1;
    if (pl == DST_PLAN_AUTO) pl = nslabs >= kAutoWideSlabs ? DST_PLAN_THROUGHPUT : p.plan1;
    return (pl == DST_PLAN_THROUGHPUT && p.Wt && N < 1024) ? 1 : 0;
}
// Run the call with the plan as a compile-time constant PLN (0 latency, 1 throughput).
#define IBPM_PLAN_SWITCH(N, pl, ...)                                  \
    switch (pl) {                                                     \
        case 1: { constexpr int PLN = ct_plan(N, 1); __VA_ARGS__; }   \
        default: { constexpr int PLN = 0; __VA_ARGS__; }              \
    }

// The (load, emit) pairs the library uses: FP64 solves, and the three passes
// of an FP32 refinement correction.
#define IBPM_X_COMBOS(X)                                                                  \
    X(XLOAD_PLAIN, XEMIT_STORE) X(XLOAD_PLAIN, XEMIT_SUB) X(XLOAD_BC, XEMIT_STORE)       \
    X(XLOAD_BC, XEMIT_SUB) X(XLOAD_F32, XEMIT_F32) X(XLOAD_RES_LAP, XEMIT_F32)           \
    X(XLOAD_RES_A, XEMIT_F32) X(XLOAD_F32, XEMIT_ADD) X(XLOAD_F32, XEMIT_ADD_FROM)       \
    X(XLOAD_F32, XEMIT_ACC_SUB) X(XLOAD_PLAIN, XEMIT_ADD_STORE) X(XLOAD_SUM, XEMIT_STORE)                  \
    X(XLOAD_F32_SUM, XEMIT_ADD)

template <int N, int PL>
cudaError_t launch_x_p(const Geom& g, const DstPlan& px, const XPassArgs& a, cudaStream_t st) {
#define IBPM_X_DISPATCH(L, E) \
    if (a.load == L && a.emit == E) return launch_x_n<N, L, E, PL>(g, px, a, st);
    IBPM_X_COMBOS(IBPM_X_DISPATCH)
#undef IBPM_X_DISPATCH
    return cudaErrorInvalidValue;
}

template <int N>
cudaError_t launch_x_t(const Geom& g, const DstPlan& px, const XPassArgs& a, cudaStream_t st) {
    IBPM_PLAN_SWITCH(N, launch_plan(N, px, a.nslabs), return (launch_x_p<N, PLN>(g, px, a, st)))
}

template <int N, class T, int PL>
cudaError_t launch_y_n(const Geom& g, const DstPlan& py, const DstPlan& px, void* data, SlabMap map, int nslabs,
                       const SpecParams& sp, cudaStream_t st) {
    constexpr int TW = y_tile_w<N, T, PL>();
    if (g.n2 != N - 1) return cudaErrorInvalidValue;   // the tile's column stride is fixed by N
    const size_t smem = y_smem_bytes<N, T, PL>(g.n2);
    if (smem > 227 * 1024) return cudaErrorInvalidConfiguration;
    dim3 grid((g.n1 + TW - 1) / TW, nslabs);
    const int threads = y_threads<N, T, PL>();
    return launch_k(dst_y_kernel<N, T, PL>, grid, dim3(threads), smem, st, static_cast<T*>(data), map, g, py,
                    static_cast<const T*>(tabs_of<T>(px).c), sp, static_cast<T*>(nullptr), BtSynth{});
}

template <int N>
cudaError_t launch_y_t(const Geom& g, const DstPlan& py, const DstPlan& px, void* data, SlabMap map, int nslabs,
                       const SpecParams& sp, cudaStream_t st) {
    IBPM_PLAN_SWITCH(N, launch_plan(N, py, nslabs),
                     return sp.f32 ? launch_y_n<N, float, PLN>(g, py, px, data, map, nslabs, sp, st)
                                   : launch_y_n<N, double, PLN>(g, py, px, data, map, nslabs, sp, st))
}

template <int N, class T, int PL>
cudaError_t launch_ybc_n(const Geom& g, const DstPlan& py, const DstPlan& px, void* out, SlabMap map, int nslabs,
                         const SpecParams& sp, const BtSynth& bs, cudaStream_t st) {
    constexpr int TW = y_tile_w<N, T, PL>();
    if (g.n2 != N - 1) return cudaErrorInvalidValue;   // the tile's column stride is fixed by N
    const size_t smem = y_smem_bytes<N, T, PL, true>(g.n2);
    if (smem > 227 * 1024) return cudaErrorInvalidConfiguration;
    dim3 grid((g.n1 + TW - 1) / TW, nslabs);
    return launch_k(dst_y_kernel<N, T, PL, true>, grid, dim3(y_threads<N, T, PL>()), smem, st,
                    static_cast<T*>(nullptr), map, g, py, static_cast<const T*>(tabs_of<T>(px).c), sp,
                    static_cast<T*>(out), bs);
}

template <int N>
cudaError_t launch_ybc_t(const Geom& g, const DstPlan& py, const DstPlan& px, void* out, SlabMap map, int nslabs,
                         const SpecParams& sp, const BtSynth& bs, cudaStream_t st) {
    IBPM_PLAN_SWITCH(N, launch_plan(N, py, nslabs),
                     return sp.f32 ? launch_ybc_n<N, float, PLN>(g, py, px, out, map, nslabs, sp, bs, st)
                                   : launch_ybc_n<N, double, PLN>(g, py, px, out, map, nslabs, sp, bs, st))
}

template <int N, class T, int PL>
cudaError_t launch_lines_n(const Geom& g, const DstPlan& px, const void* Y, SlabMap map, int nslabs, void* smp,
                           cudaStream_t st) {
    constexpr int TP = ct_tp(N, PL);
    dim3 grid(1 + (g.ny / 2 + 1 + TP / 32 - 1) / (TP / 32), nslabs);
    return launch_k(dst_lines_kernel<N, T, PL>, grid, dim3(TP), lines_smem_bytes<N, PL>(), st,
                    static_cast<const T*>(Y), map, g, px, static_cast<double*>(smp));
}

template <int N>
cudaError_t launch_lines_t(const Geom& g, const DstPlan& px, const void* Y, SlabMap map, int nslabs, void* smp,
                           int f32, cudaStream_t st) {
    IBPM_PLAN_SWITCH(N, launch_plan(N, px, 1),
                     return f32 ? launch_lines_n<N, float, PLN>(g, px, Y, map, nslabs, smp, st)
                                : launch_lines_n<N, double, PLN>(g, px, Y, map, nslabs, smp, st))
}

template <class K>
cudaError_t smem_attrs(K kernel) {
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
    if (e != cudaSuccess) return e;
    // the largest shared-memory carveout, so that occupancy is not capped by L1
    return cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
}

template <int N, int PL>
cudaError_t attr_plan() {
    cudaError_t e;
#define IBPM_X_ATTR(L, E) \
    if ((e = smem_attrs(dst_x_kernel<N, L, E, PL>))) return e;
    IBPM_X_COMBOS(IBPM_X_ATTR)
#undef IBPM_X_ATTR
    if ((e = smem_attrs(dst_y_kernel<N, double, PL>))) return e;
    if ((e = smem_attrs(dst_y_kernel<N, double, PL, true>))) return e;
    if ((e = smem_attrs(dst_y_kernel<N, float, PL, true>))) return e;
    if ((e = smem_attrs(dst_lines_kernel<N, double, PL>))) return e;
    if ((e = smem_attrs(dst_lines_kernel<N, float, PL>))) return e;
    return smem_attrs(dst_y_kernel<N, float, PL>);
}

template <int N>
cudaError_t attr_t() {
    cudaError_t e = attr_plan<N, 0>();
    if (e != cudaSuccess || ct_plan(N, 1) == 0) return e;
    return attr_plan<N, ct_plan(N, 1)>();
}

}  // namespace dstk

// Non-template entry points for one length, defined in one translation unit
// per length (dst_n<N>.cu) so the lengths compile in parallel.
#define IBPM_DST_DEFINE(N)                                                                                 \
    cudaError_t dst_x_##N(const Geom& g, const DstPlan& px, const XPassArgs& a, cudaStream_t st) {         \
        return dstk::launch_x_t<N>(g, px, a, st);                                                          \
    }                                                                                                      \
    cudaError_t dst_y_##N(const Geom& g, const DstPlan& py, const DstPlan& px, void* d, SlabMap m, int n,   \
                          const SpecParams& sp, cudaStream_t st) {                                         \
        return dstk::launch_y_t<N>(g, py, px, d, m, n, sp, st);                                            \
    }                                                                                                      \
    cudaError_t dst_attr_##N() { return dstk::attr_t<N>(); }                                               \
    cudaError_t dst_ybc_##N(const Geom& g, const DstPlan& py, const DstPlan& px, void* o, SlabMap m, int n,  \
                            const SpecParams& sp, const BtSynth& bs, cudaStream_t st) {                     \
        return dstk::launch_ybc_t<N>(g, py, px, o, m, n, sp, bs, st);                                      \
    }                                                                                                      \
    cudaError_t dst_lines_##N(const Geom& g, const DstPlan& px, const void* Y, SlabMap m, int n, void* smp, \
                              int f32, cudaStream_t st) {                                                  \
        return dstk::launch_lines_t<N>(g, px, Y, m, n, smp, f32, st);                                      \
    }

}  // namespace ibpm
