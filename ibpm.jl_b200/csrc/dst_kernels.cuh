// Batched 2-D DST-I (FFTW RODFT00, unnormalised) for the Poisson-type solves of
// the IBPM step: x = S((S b) ./ M .* scale), S the 2-D DST-I
// (src/fluid-operators/dst-inversion.jl:145-156, laplacian.jl:180-232).
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
// The FFT is a mixed-radix (8, 5, 4, 3, 2) Stockham transform, run in place in
// shared memory by one "group" of TP = N/8 threads (at least one warp): each
// stage reads all its inputs into registers, synchronises the group, then
// writes.  N is a template parameter, so every stride, radix and loop bound is
// a compile-time constant.  Shared-memory indices are padded by one element
// every eight (pad(i) = i + i/8) so the stride-8 writes of the first stage are
// free of bank conflicts.
#pragma once

#include "ibpm_internal.cuh"

namespace ibpm {
namespace dstk {

__host__ __device__ constexpr int ct_radix(int N, int s) {
    int n = N, idx = 0;
    const int rs[5] = {8, 5, 4, 3, 2};
    for (int i = 0; i < 5; ++i) {
        while (n % rs[i] == 0) {
            if (idx == s) return rs[i];
            n /= rs[i];
            ++idx;
        }
    }
    return 1;
}
__host__ __device__ constexpr int ct_nstages(int N) {
    int n = N, s = 0;
    const int rs[5] = {8, 5, 4, 3, 2};
    for (int i = 0; i < 5; ++i)
        while (n % rs[i] == 0) { n /= rs[i]; ++s; }
    return n == 1 ? s : -1;
}
__host__ __device__ constexpr int ct_tp(int N) {
    int t = ((N / 8 + 31) / 32) * 32;
    return t < 32 ? 32 : t;
}
__host__ __device__ constexpr int ct_pad(int i) { return i + (i >> 3); }
__host__ __device__ constexpr int ct_buf(int N) { return ct_pad(N) + 8; }  // + scan scratch

__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cmuli(double2 a) { return make_double2(-a.y, a.x); }  // i·a

// Small DFTs with the +2πi sign: V_b = Σ_a v_a e^{+2πi ab/R}.
template <int R> __device__ __forceinline__ void dft(double2* v);

template <> __device__ __forceinline__ void dft<2>(double2* v) {
    const double2 t = v[0];
    v[0] = cadd(t, v[1]);
    v[1] = csub(t, v[1]);
}

template <> __device__ __forceinline__ void dft<3>(double2* v) {
    const double h3 = 0.86602540378443864676;  // √3 / 2
    const double2 s = cadd(v[1], v[2]);
    const double2 d = csub(v[1], v[2]);
    const double2 a = make_double2(v[0].x - 0.5 * s.x, v[0].y - 0.5 * s.y);
    const double2 b = make_double2(-h3 * d.y, h3 * d.x);  // i (√3/2) d
    v[0] = cadd(v[0], s);
    v[1] = cadd(a, b);
    v[2] = csub(a, b);
}

template <> __device__ __forceinline__ void dft<4>(double2* v) {
    const double2 t0 = cadd(v[0], v[2]);
    const double2 t1 = csub(v[0], v[2]);
    const double2 t2 = cadd(v[1], v[3]);
    const double2 t3 = cmuli(csub(v[1], v[3]));
    v[0] = cadd(t0, t2);
    v[2] = csub(t0, t2);
    v[1] = cadd(t1, t3);
    v[3] = csub(t1, t3);
}

template <> __device__ __forceinline__ void dft<5>(double2* v) {
    const double c1 = 0.30901699437494742410;   // cos(2π/5)
    const double c2 = -0.80901699437494742410;  // cos(4π/5)
    const double s1 = 0.95105651629515357212;   // sin(2π/5)
    const double s2 = 0.58778525229247312917;   // sin(4π/5)
    const double2 s14 = cadd(v[1], v[4]), d14 = csub(v[1], v[4]);
    const double2 s23 = cadd(v[2], v[3]), d23 = csub(v[2], v[3]);
    const double2 a1 = make_double2(v[0].x + c1 * s14.x + c2 * s23.x, v[0].y + c1 * s14.y + c2 * s23.y);
    const double2 a2 = make_double2(v[0].x + c2 * s14.x + c1 * s23.x, v[0].y + c2 * s14.y + c1 * s23.y);
    const double2 b1 = cmuli(make_double2(s1 * d14.x + s2 * d23.x, s1 * d14.y + s2 * d23.y));
    const double2 b2 = cmuli(make_double2(s2 * d14.x - s1 * d23.x, s2 * d14.y - s1 * d23.y));
    v[0] = cadd(v[0], cadd(s14, s23));
    v[1] = cadd(a1, b1);
    v[4] = csub(a1, b1);
    v[2] = cadd(a2, b2);
    v[3] = csub(a2, b2);
}

template <> __device__ __forceinline__ void dft<8>(double2* v) {
    const double r2 = 0.70710678118654752440;  // √2 / 2
    double2 e[4] = {v[0], v[2], v[4], v[6]};
    double2 o[4] = {v[1], v[3], v[5], v[7]};
    dft<4>(e);
    dft<4>(o);
    o[1] = make_double2(r2 * (o[1].x - o[1].y), r2 * (o[1].x + o[1].y));    // × e^{iπ/4}
    o[2] = cmuli(o[2]);                                                    // × i
    o[3] = make_double2(-r2 * (o[3].x + o[3].y), r2 * (o[3].x - o[3].y));  // × e^{3iπ/4}
#pragma unroll
    for (int b = 0; b < 4; ++b) {
        v[b] = cadd(e[b], o[b]);
        v[b + 4] = csub(e[b], o[b]);
    }
}

// Synchronise the TP threads of group `gid` (named barrier 1 + gid when the
// group spans several warps).
template <int TP> __device__ __forceinline__ void gsync(int gid) {
    if constexpr (TP == 32) {
        __syncwarp();
    } else {
        asm volatile("bar.sync %0, %1;" ::"r"(gid + 1), "n"(TP) : "memory");
    }
}

template <int N, int TP, int R, int Ns>
__device__ __forceinline__ void fft_stage(double2* buf, const double2* __restrict__ W, int tid, int gid) {
    constexpr int nb = N / R;
    constexpr int QM = (nb + TP - 1) / TP;
    constexpr bool exact = (QM * TP == nb);
    constexpr int ts = N / (Ns * R);
    double2 v[QM][R];
#pragma unroll
    for (int q = 0; q < QM; ++q) {
        const int b = tid + q * TP;
        if (exact || b < nb) {
#pragma unroll
            for (int r = 0; r < R; ++r) v[q][r] = buf[ct_pad(b + r * nb)];
        }
    }
    gsync<TP>(gid);
#pragma unroll
    for (int q = 0; q < QM; ++q) {
        const int b = tid + q * TP;
        if (exact || b < nb) {
            const int k = b % Ns;
            if constexpr (Ns > 1) {
#pragma unroll
                for (int r = 1; r < R; ++r) v[q][r] = cmul(v[q][r], __ldg(&W[k * r * ts]));
            }
            dft<R>(v[q]);
            const int base = (b - k) * R + k;
#pragma unroll
            for (int r = 0; r < R; ++r) buf[ct_pad(base + r * Ns)] = v[q][r];
        }
    }
    gsync<TP>(gid);
}

template <int N, int TP, int S, int Ns>
__device__ __forceinline__ void fft_stages(double2* buf, const double2* __restrict__ W, int tid, int gid) {
    if constexpr (S < ct_nstages(N)) {
        constexpr int R = ct_radix(N, S);
        fft_stage<N, TP, R, Ns>(buf, W, tid, gid);
        fft_stages<N, TP, S + 1, Ns * R>(buf, W, tid, gid);
    }
}

// Pre-processing: buf[m] = y_m from load(m-1) = (a_{m-1}, b_{m-1}).
template <int N, int TP, class Load>
__device__ __forceinline__ void dst_pre(double2* buf, const double* __restrict__ s, int tid, Load load) {
    constexpr int half = N >> 1;
    for (int m = tid; m <= half; m += TP) {
        if (m == 0) {
            buf[0] = make_double2(0.0, 0.0);
            continue;
        }
        const double2 fm = load(m - 1);
        if (m == half) {  // sin(π/2) = 1
            buf[ct_pad(m)] = make_double2(2.0 * fm.x, 2.0 * fm.y);
            continue;
        }
        const double2 fn = load(N - m - 1);
        const double sm = __ldg(&s[m]);
        const double2 sum = cadd(fm, fn), dif = csub(fm, fn);
        const double2 ys = make_double2(sm * sum.x, sm * sum.y);
        buf[ct_pad(m)] = make_double2(ys.x + 0.5 * dif.x, ys.y + 0.5 * dif.y);
        buf[ct_pad(N - m)] = make_double2(ys.x - 0.5 * dif.x, ys.y - 0.5 * dif.y);
    }
}

__device__ __forceinline__ double2 shfl_up2(double2 v, int off) {
    return make_double2(__shfl_up_sync(0xffffffffu, v.x, off), __shfl_up_sync(0xffffffffu, v.y, off));
}

// Exclusive prefix sum of one double2 per thread over the TP threads of a group.
template <int TP>
__device__ __forceinline__ double2 group_excl_scan(double2 v, int tid, int gid, double2* scratch) {
    const int lane = tid & 31, w = tid >> 5;
    double2 inc = v;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const double2 n = shfl_up2(inc, off);
        if (lane >= off) inc = cadd(inc, n);
    }
    double2 ex = shfl_up2(inc, 1);
    if (lane == 0) ex = make_double2(0.0, 0.0);
    if constexpr (TP > 32) {
        if (lane == 31) scratch[w] = inc;
        gsync<TP>(gid);
        double2 base = make_double2(0.0, 0.0);
        for (int u = 0; u < w; ++u) base = cadd(base, scratch[u]);
        ex = cadd(base, ex);
    }
    return ex;
}

// Post-processing: from Z (in buf) produce the N-1 outputs of both lines and
// hand them to emit(o, (a_o, b_o)).  All reads of buf precede every emit, so
// emit may write into buf.
template <int N, int TP, class Emit>
__device__ __forceinline__ void dst_post(double2* buf, int tid, int gid, double2* scratch, Emit emit) {
    constexpr int half = N >> 1;
    constexpr int C = (half + TP - 1) / TP;
    const int k0 = tid * C;
    double2 D[C], O[C];
    double2 tot = make_double2(0.0, 0.0);
#pragma unroll
    for (int t = 0; t < C; ++t) {
        const int k = k0 + t;
        if (k < half) {
            const double2 zk = buf[ct_pad(k)];
            double2 d;
            if (k == 0) {
                d = zk;
                O[t] = make_double2(0.0, 0.0);
            } else {
                const double2 zn = buf[ct_pad(N - k)];
                d = cadd(zk, zn);
                const double2 dl = csub(zk, zn);
                O[t] = make_double2(dl.y, -dl.x);  // −i (Z_k − Z_{N−k})
            }
            tot = cadd(tot, d);
            D[t] = tot;
        }
    }
    const double2 ex = group_excl_scan<TP>(tot, tid, gid, scratch);
    gsync<TP>(gid);
#pragma unroll
    for (int t = 0; t < C; ++t) {
        const int k = k0 + t;
        if (k < half) {
            emit(2 * k, cadd(ex, D[t]));
            if (k > 0) emit(2 * k - 1, O[t]);
        }
    }
}

// One DST-I of a line pair: load → pre → FFT → post → emit.
template <int N, int TP, class Load, class Emit>
__device__ __forceinline__ void dst_pair(double2* buf, const double2* __restrict__ W, const double* __restrict__ s,
                                         int tid, int gid, Load load, Emit emit) {
    dst_pre<N, TP>(buf, s, tid, load);
    gsync<TP>(gid);
    fft_stages<N, TP, 0, 1>(buf, W, tid, gid);
    dst_post<N, TP>(buf, tid, gid, buf + ct_pad(N), emit);
}

// ---------------------------------------------------------------------------
// x-pass: lines are rows of a slab (contiguous).  One group per line pair.
// ---------------------------------------------------------------------------
template <int N, int LOAD, int EMIT>
__global__ void __launch_bounds__(256) dst_x_kernel(XPassArgs a, Geom g, const double2* __restrict__ W,
                                                    const double* __restrict__ s) {
    constexpr int TP = ct_tp(N);
    constexpr int G = 256 / TP;
    extern __shared__ double2 smem2[];
    const int gid = threadIdx.x / TP, tid = threadIdx.x % TP;
    double2* buf = smem2 + gid * ct_buf(N);
    const int la = a.line0 + 2 * (blockIdx.x * G + gid);
    if (la >= a.line1) return;  // the whole group leaves together
    const bool hasb = (la + 1) < a.line1;
    const int y = blockIdx.y;
    const int P = g.P, n1 = g.n1, n2 = g.n2;
    const double* ra = a.in + a.in_map.off(y) + (long long)la * P;
    const double* rb = ra + P;

    CoarseBC cb;
    cb.rc = nullptr; cb.P = P; cb.nx = g.nx; cb.ny = g.ny;
    if (LOAD == XLOAD_BC && a.coarse) cb.rc = a.coarse + a.coarse_map.off(y);

    // apply_bc!(r, get_bc!(coarse), 1.0) (mg-utils.jl:43-60) in the reference's
    // order: bottom row, top row, left column, right column.
    auto with_bc = [&](double v, int i, int j) -> double {
        if (j == 0) v += cb.bot(i + 1);
        if (j == n2 - 1) v += cb.top(i + 1);
        if (i == 0) v += cb.left(j + 1);
        if (i == n1 - 1) v += cb.right(j + 1);
        return v;
    };
    auto load = [&](int i) -> double2 {
        double va = ra[i];
        double vb = hasb ? rb[i] : 0.0;
        if (LOAD == XLOAD_BC && cb.rc) {
            va = with_bc(va, i, la);
            if (hasb) vb = with_bc(vb, i, la + 1);
        }
        return make_double2(va, vb);
    };
    dst_pair<N, TP>(buf, W, s, tid, gid, load, [&](int o, double2 v) { buf[ct_pad(o)] = v; });
    gsync<TP>(gid);
    double* oa = a.out + a.out_map.off(y) + (long long)la * P;
    double* ob = oa + P;
    for (int o = tid; o < n1; o += TP) {
        const double2 v = buf[ct_pad(o)];
        if (EMIT == XEMIT_STORE) {
            oa[o] = v.x;
            if (hasb) ob[o] = v.y;
        } else {
            oa[o] -= v.x;
            if (hasb) ob[o] -= v.y;
        }
    }
}

// ---------------------------------------------------------------------------
// y-pass of a Poisson solve: DST-I along y, spectral divide, DST-I along y,
// in place on a tile of TW = 2G columns (all rows) staged in shared memory.
// ---------------------------------------------------------------------------
template <int N>
__host__ __device__ constexpr int y_tile_w() { return 2 * (256 / ct_tp(N)); }
template <int N>
__host__ __device__ constexpr size_t y_smem_bytes(int n2) {
    return (size_t)(((n2 * (y_tile_w<N>() + 1) + 1) / 2) * 2) * sizeof(double) +
           (size_t)(256 / ct_tp(N)) * ct_buf(N) * sizeof(double2);
}

template <int N>
__global__ void __launch_bounds__(256) dst_y_solve_kernel(double* data, SlabMap map, Geom g,
                                                          const double2* __restrict__ W, const double* __restrict__ s,
                                                          const double* __restrict__ cy,
                                                          const double* __restrict__ cx, SpecParams sp) {
    constexpr int TP = ct_tp(N);
    constexpr int TW = y_tile_w<N>();
    constexpr int TWp = TW + 1;
    extern __shared__ double smemd[];
    const int gid = threadIdx.x / TP, tid = threadIdx.x % TP;
    const int P = g.P, n1 = g.n1, n2 = g.n2;
    double* tile = smemd;
    const int tile_d = ((n2 * TWp + 1) / 2) * 2;
    double2* buf = reinterpret_cast<double2*>(smemd + tile_d) + gid * ct_buf(N);
    const int i0 = blockIdx.x * TW;
    double* base = data + map.off(blockIdx.y);
    const int lev = map.level(blockIdx.y);

    for (int idx = threadIdx.x; idx < n2 * TW; idx += blockDim.x) {
        const int j = idx / TW, c = idx - j * TW;
        const int i = i0 + c;
        tile[j * TWp + c] = (i < n1) ? base[(long long)j * P + i] : 0.0;
    }
    __syncthreads();

    const int ca = 2 * gid;
    const int ia = i0 + ca;
    if (ia < n1) {
        auto load = [&](int m) -> double2 { return make_double2(tile[m * TWp + ca], tile[m * TWp + ca + 1]); };
        auto emit = [&](int o, double2 v) {
            tile[o * TWp + ca] = v.x;
            tile[o * TWp + ca + 1] = v.y;
        };
        dst_pair<N, TP>(buf, W, s, tid, gid, load, emit);
        gsync<TP>(gid);
        // w ./= M ; w .*= scale  with Λ = -2 (cos(π i/nx) + cos(π j/ny) - 2)
        const bool hasb = ia + 1 < n1;
        const double cxa = __ldg(&cx[ia]);
        const double cxb = hasb ? __ldg(&cx[ia + 1]) : 0.0;
        const double den = sp.den[lev];
        for (int o = tid; o < n2; o += TP) {
            const double c2 = __ldg(&cy[o]);
            const double la = -2.0 * ((cxa + c2) - 2.0);
            const double lb = -2.0 * ((cxb + c2) - 2.0);
            double Ma, Mb;
            if (sp.mode == SPEC_DELTA) {
                Ma = la;
                Mb = lb;
            } else {
                Ma = 1.0 + la * sp.dt / den;
                Mb = 1.0 + lb * sp.dt / den;
            }
            tile[o * TWp + ca] = (tile[o * TWp + ca] / Ma) * sp.scale;
            tile[o * TWp + ca + 1] = hasb ? (tile[o * TWp + ca + 1] / Mb) * sp.scale : 0.0;
        }
        gsync<TP>(gid);
        dst_pair<N, TP>(buf, W, s, tid, gid, load, emit);
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < n2 * TW; idx += blockDim.x) {
        const int j = idx / TW, c = idx - j * TW;
        const int i = i0 + c;
        if (i < n1) base[(long long)j * P + i] = tile[j * TWp + c];
    }
}

// ---------------------------------------------------------------------------
// Launchers for one compile-time length.
// ---------------------------------------------------------------------------
template <int N, int LOAD, int EMIT>
cudaError_t launch_x_n(const Geom& g, const DstPlan& px, const XPassArgs& a, cudaStream_t st) {
    constexpr int TP = ct_tp(N);
    constexpr int G = 256 / TP;
    const int lines = a.line1 - a.line0;
    if (lines <= 0 || a.nslabs <= 0) return cudaSuccess;
    const int pairs = (lines + 1) / 2;
    dim3 grid((pairs + G - 1) / G, a.nslabs);
    const size_t smem = (size_t)G * ct_buf(N) * sizeof(double2);
    dst_x_kernel<N, LOAD, EMIT><<<grid, G * TP, smem, st>>>(a, g, px.W, px.s);
    return cudaGetLastError();
}

template <int N>
cudaError_t launch_x_t(const Geom& g, const DstPlan& px, const XPassArgs& a, cudaStream_t st) {
    if (a.load == XLOAD_BC)
        return a.emit == XEMIT_SUB ? launch_x_n<N, XLOAD_BC, XEMIT_SUB>(g, px, a, st)
                                   : launch_x_n<N, XLOAD_BC, XEMIT_STORE>(g, px, a, st);
    return a.emit == XEMIT_SUB ? launch_x_n<N, XLOAD_PLAIN, XEMIT_SUB>(g, px, a, st)
                               : launch_x_n<N, XLOAD_PLAIN, XEMIT_STORE>(g, px, a, st);
}

template <int N>
cudaError_t launch_y_t(const Geom& g, const DstPlan& py, const DstPlan& px, double* data, SlabMap map, int nslabs,
                       const SpecParams& sp, cudaStream_t st) {
    constexpr int TW = y_tile_w<N>();
    const size_t smem = y_smem_bytes<N>(g.n2);
    if (smem > 227 * 1024) return cudaErrorInvalidConfiguration;
    dim3 grid((g.n1 + TW - 1) / TW, nslabs);
    dst_y_solve_kernel<N><<<grid, 256, smem, st>>>(data, map, g, py.W, py.s, py.c, px.c, sp);
    return cudaGetLastError();
}

template <int N>
cudaError_t attr_t() {
    const int big = 227 * 1024;
    cudaError_t e;
    if ((e = cudaFuncSetAttribute(dst_x_kernel<N, XLOAD_PLAIN, XEMIT_STORE>, cudaFuncAttributeMaxDynamicSharedMemorySize, big))) return e;
    if ((e = cudaFuncSetAttribute(dst_x_kernel<N, XLOAD_PLAIN, XEMIT_SUB>, cudaFuncAttributeMaxDynamicSharedMemorySize, big))) return e;
    if ((e = cudaFuncSetAttribute(dst_x_kernel<N, XLOAD_BC, XEMIT_STORE>, cudaFuncAttributeMaxDynamicSharedMemorySize, big))) return e;
    if ((e = cudaFuncSetAttribute(dst_x_kernel<N, XLOAD_BC, XEMIT_SUB>, cudaFuncAttributeMaxDynamicSharedMemorySize, big))) return e;
    return cudaFuncSetAttribute(dst_y_solve_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
}

}  // namespace dstk

// Non-template entry points for one length, defined in one translation unit
// per length (dst_n<N>.cu) so the lengths compile in parallel.
#define IBPM_DST_DEFINE(N)                                                                                 \
    cudaError_t dst_x_##N(const Geom& g, const DstPlan& px, const XPassArgs& a, cudaStream_t st) {         \
        return dstk::launch_x_t<N>(g, px, a, st);                                                          \
    }                                                                                                      \
    cudaError_t dst_y_##N(const Geom& g, const DstPlan& py, const DstPlan& px, double* d, SlabMap m, int n, \
                          const SpecParams& sp, cudaStream_t st) {                                         \
        return dstk::launch_y_t<N>(g, py, px, d, m, n, sp, st);                                            \
    }                                                                                                      \
    cudaError_t dst_attr_##N() { return dstk::attr_t<N>(); }

}  // namespace ibpm
