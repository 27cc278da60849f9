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

// Twiddles of stage S (sub-transform length Ns before it, radix R) are stored
// contiguously as T[(r-1)·Ns + k] = exp(+2πi k r/(Ns R)), r = 1…R-1, k < Ns, so
// the threads of a stage (consecutive k) read consecutive entries.
__host__ __device__ constexpr int ct_stage_ns(int N, int S) {
    int ns = 1;
    for (int s = 0; s < S; ++s) ns *= ct_radix(N, s);
    return ns;
}
__host__ __device__ constexpr int ct_tw_off(int N, int S) {
    int off = 0;
    for (int s = 0; s < S; ++s) {
        const int ns = ct_stage_ns(N, s);
        if (ns > 1) off += (ct_radix(N, s) - 1) * ns;
    }
    return off;
}
__host__ __device__ constexpr int ct_tw_count(int N) { return ct_tw_off(N, ct_nstages(N)); }
// Groups (line pairs) per CTA: 128-thread CTAs for N <= 1024.
__host__ __device__ constexpr int ct_groups(int N) { return ct_tp(N) >= 128 ? 1 : 128 / ct_tp(N); }

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
// The barrier id is an immediate in each branch, so ptxas reserves only the
// barriers a kernel can use (a run-time id reserves all sixteen, which caps
// the resident blocks per SM).
template <int TP> __device__ __forceinline__ void gsync(int gid) {
    if constexpr (TP == 32) {
        __syncwarp();
    } else if constexpr (TP >= 128) {
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

template <int N, int TP, int R, int Ns, int TWOFF>
__device__ __forceinline__ void fft_stage(double2* buf, const double2* W, int tid, int gid) {
    constexpr int nb = N / R;
    constexpr int QM = (nb + TP - 1) / TP;
    constexpr bool exact = (QM * TP == nb);
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
                for (int r = 1; r < R; ++r) v[q][r] = cmul(v[q][r], W[TWOFF + (r - 1) * Ns + k]);
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
__device__ __forceinline__ void fft_stages(double2* buf, const double2* W, int tid, int gid) {
    if constexpr (S < ct_nstages(N)) {
        constexpr int R = ct_radix(N, S);
        fft_stage<N, TP, R, Ns, ct_tw_off(N, S)>(buf, W, tid, gid);
        fft_stages<N, TP, S + 1, Ns * R>(buf, W, tid, gid);
    }
}

// Pre-processing: buf[m] = y_m from load(m-1) = (a_{m-1}, b_{m-1}).
template <int N, int TP, class Load>
__device__ __forceinline__ void dst_pre(double2* buf, const double* s, int tid, Load load) {
    constexpr int half = N >> 1;
    constexpr int IT = (half + TP) / TP;  // m = tid + it·TP covers 0 … half
    double2 fm[IT], fn[IT];
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
            buf[0] = make_double2(0.0, 0.0);
        } else if (m == half) {  // sin(π/2) = 1
            buf[ct_pad(m)] = make_double2(2.0 * fm[it].x, 2.0 * fm[it].y);
        } else if (m < half) {
            const double sm = s[m];
            const double2 sum = cadd(fm[it], fn[it]), dif = csub(fm[it], fn[it]);
            const double2 ys = make_double2(sm * sum.x, sm * sum.y);
            buf[ct_pad(m)] = make_double2(ys.x + 0.5 * dif.x, ys.y + 0.5 * dif.y);
            buf[ct_pad(N - m)] = make_double2(ys.x - 0.5 * dif.x, ys.y - 0.5 * dif.y);
        }
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
__device__ __forceinline__ void dst_pair(double2* buf, const double2* W, const double* s, int tid, int gid, Load load,
                                         Emit emit) {
    dst_pre<N, TP>(buf, s, tid, load);
    gsync<TP>(gid);
    fft_stages<N, TP, 0, 1>(buf, W, tid, gid);
    dst_post<N, TP>(buf, tid, gid, buf + ct_pad(N), emit);
}

// Copy the transform tables into shared memory: stage twiddles (complex),
// then sin(πm/N) for m ≤ N/2.
template <int N>
__device__ __forceinline__ void stage_tables(double2* tw, double* sn, const DstPlan& p) {
    for (int i = threadIdx.x; i < ct_tw_count(N); i += blockDim.x) cp_async16(tw + i, p.W + i);
    for (int i = threadIdx.x; i <= N / 2; i += blockDim.x) cp_async8(sn + i, p.s + i);
}
template <int N>
__host__ __device__ constexpr size_t tables_bytes() {
    return (size_t)ct_tw_count(N) * sizeof(double2) + (size_t)((N / 2 + 2) & ~1) * sizeof(double);
}

// ---------------------------------------------------------------------------
// x-pass: lines are rows of a slab (contiguous).  One group per line pair.
// ---------------------------------------------------------------------------
template <int N, int LOAD, int EMIT>
__global__ void __launch_bounds__((N <= 1024 ? 128 : 256)) dst_x_kernel(XPassArgs a, Geom g, DstPlan p) {
    constexpr int TP = ct_tp(N);
    constexpr int G = ct_groups(N);
    extern __shared__ double2 smem2[];
    double2* tw = smem2;
    double* sn = reinterpret_cast<double*>(smem2 + ct_tw_count(N));
    double2* bufs = reinterpret_cast<double2*>(reinterpret_cast<char*>(smem2) + tables_bytes<N>());
    stage_tables<N>(tw, sn, p);  // constant tables: before the dependency wait
    cp_async_wait();
    __syncthreads();
    pdl_wait();
    pdl_trigger();
    const int gid = threadIdx.x / TP, tid = threadIdx.x % TP;
    double2* buf = bufs + gid * ct_buf(N);
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
    dst_pair<N, TP>(buf, tw, sn, tid, gid, load, [&](int o, double2 v) { buf[ct_pad(o)] = v; });
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
// y-pass of a Poisson-type solve on a tile of TW = 2G columns (all rows)
// staged in shared memory, in place: DST-I, spectral divide, DST-I.
// ---------------------------------------------------------------------------
template <int N>
__host__ __device__ constexpr int y_groups() { return ct_groups(N); }
template <int N>
__host__ __device__ constexpr int y_tile_w() { return 2 * y_groups<N>(); }
template <int N>
__host__ __device__ constexpr size_t y_smem_bytes(int n2) {
    return tables_bytes<N>() + (size_t)(((n2 + 1) / 2) * 2) * sizeof(double) +  // cos(π(j+1)/ny)
           (size_t)(((n2 * (y_tile_w<N>() + 1) + 1) / 2) * 2) * sizeof(double) +
           (size_t)y_groups<N>() * ct_buf(N) * sizeof(double2);
}

template <int N>
__global__ void __launch_bounds__((N <= 1024 ? 128 : 256), (N <= 512 ? 5 : 1))
    dst_y_kernel(double* data, SlabMap map, Geom g, DstPlan p, const double* __restrict__ cx, SpecParams sp) {
    constexpr int TP = ct_tp(N);
    constexpr int TW = y_tile_w<N>();
    constexpr int TWp = TW + 1;
    extern __shared__ double2 smem2[];
    const int P = g.P, n1 = g.n1, n2 = g.n2;
    double2* tw = smem2;
    double* sn = reinterpret_cast<double*>(smem2 + ct_tw_count(N));
    double* cyv = reinterpret_cast<double*>(reinterpret_cast<char*>(smem2) + tables_bytes<N>());
    double* tile = cyv + ((n2 + 1) / 2) * 2;
    const int tile_d = ((n2 * TWp + 1) / 2) * 2;
    const int gid = threadIdx.x / TP, tid = threadIdx.x % TP;
    double2* buf = reinterpret_cast<double2*>(tile + tile_d) + gid * ct_buf(N);
    const int i0 = blockIdx.x * TW;
    double* base = data + map.off(blockIdx.y);
    const int lev = map.level(blockIdx.y);

    stage_tables<N>(tw, sn, p);  // constant tables: before the dependency wait
    for (int j = threadIdx.x; j < n2; j += blockDim.x) cp_async8(cyv + j, p.c + j);
    pdl_wait();
    pdl_trigger();
    for (int idx = threadIdx.x; idx < n2 * TW; idx += blockDim.x) {
        const int j = idx / TW, c = idx - j * TW;
        const int i = i0 + c;
        if (i < n1) cp_async8(tile + j * TWp + c, base + (long long)j * P + i);
        else tile[j * TWp + c] = 0.0;
    }
    cp_async_wait();
    __syncthreads();

    const int ca = 2 * gid;
    const int ia = i0 + ca;
    if (ia < n1) {
        const bool hasb = ia + 1 < n1;
        auto load = [&](int m) -> double2 { return make_double2(tile[m * TWp + ca], tile[m * TWp + ca + 1]); };
        auto emit = [&](int o, double2 v) {
            tile[o * TWp + ca] = v.x;
            tile[o * TWp + ca + 1] = v.y;
        };
        // w ./= M ; w .*= scale  with Λ = -2 (cos(π i/nx) + cos(π j/ny) - 2)
        auto divide = [&]() {
            const double cxa = __ldg(&cx[ia]);
            const double cxb = hasb ? __ldg(&cx[ia + 1]) : 0.0;
            const double den = sp.den[lev];
            for (int o = tid; o < n2; o += TP) {
                const double c2 = cyv[o];
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
                tile[o * TWp + ca] = (tile[o * TWp + ca] * nr_rcp(Ma)) * sp.scale;
                tile[o * TWp + ca + 1] = hasb ? (tile[o * TWp + ca + 1] * nr_rcp(Mb)) * sp.scale : 0.0;
            }
        };
        dst_pair<N, TP>(buf, tw, sn, tid, gid, load, emit);
        gsync<TP>(gid);
        divide();
        gsync<TP>(gid);
        dst_pair<N, TP>(buf, tw, sn, tid, gid, load, emit);
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
    constexpr int G = ct_groups(N);
    const int lines = a.line1 - a.line0;
    if (lines <= 0 || a.nslabs <= 0) return cudaSuccess;
    const int pairs = (lines + 1) / 2;
    dim3 grid((pairs + G - 1) / G, a.nslabs);
    const size_t smem = tables_bytes<N>() + (size_t)G * ct_buf(N) * sizeof(double2);
    return launch_k(dst_x_kernel<N, LOAD, EMIT>, grid, dim3(G * TP), smem, st, a, g, px);
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
    const int threads = y_groups<N>() * ct_tp(N);
    return launch_k(dst_y_kernel<N>, grid, dim3(threads), smem, st, data, map, g, py, px.c, sp);
}

template <class K>
cudaError_t smem_attrs(K kernel) {
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
    if (e != cudaSuccess) return e;
    // the largest shared-memory carveout, so that occupancy is not capped by L1
    return cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
}

template <int N>
cudaError_t attr_t() {
    cudaError_t e;
    if ((e = smem_attrs(dst_x_kernel<N, XLOAD_PLAIN, XEMIT_STORE>))) return e;
    if ((e = smem_attrs(dst_x_kernel<N, XLOAD_PLAIN, XEMIT_SUB>))) return e;
    if ((e = smem_attrs(dst_x_kernel<N, XLOAD_BC, XEMIT_STORE>))) return e;
    if ((e = smem_attrs(dst_x_kernel<N, XLOAD_BC, XEMIT_SUB>))) return e;
    return smem_attrs(dst_y_kernel<N>);
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
