// Transform tables and length dispatch of the batched DST-I kernels
// (kernels: dst_kernels.cuh, one instantiation unit per length: dst_n<N>.cu).
#include "dst_kernels.cuh"

#include <math.h>

namespace ibpm {


// Every supported transform length N = nx or ny.
#define IBPM_DST_LENGTHS(X) X(32) X(64) X(128) X(192) X(200) X(256) X(384) X(400) X(512) X(768) X(1024) X(2048)

#define IBPM_DST_DECLARE(N)                                                                                   \
    cudaError_t dst_x_##N(const Geom&, const DstPlan&, const XPassArgs&, cudaStream_t);                      \
    cudaError_t dst_y_##N(const Geom&, const DstPlan&, const DstPlan&, void*, SlabMap, int, const SpecParams&, \
                          cudaStream_t);                                                                     \
    cudaError_t dst_attr_##N();                                                                              \
    cudaError_t dst_ybc_##N(const Geom&, const DstPlan&, const DstPlan&, void*, SlabMap, int, const SpecParams&, \
                            const BtSynth&, cudaStream_t);                                                   \
    cudaError_t dst_lines_##N(const Geom&, const DstPlan&, const void*, SlabMap, int, void*, int, cudaStream_t);
IBPM_DST_LENGTHS(IBPM_DST_DECLARE)
#undef IBPM_DST_DECLARE

// Supported transform lengths N = nx or ny: 32, 64, 128, 192, 200, 256, 384, 400, 512, 768, 1024, 2048.
bool dst_supported(int N) {
    switch (N) {
#define IBPM_CASE(L) case L:
        IBPM_DST_LENGTHS(IBPM_CASE)
#undef IBPM_CASE
            return true;
        default:
            return false;
    }
}

// Stage layout of the length-N FFT, for the twiddle table kernel.
struct StageDesc {
    int n;
    int ns[8], r[8], off[8];
};

static StageDesc stage_desc(int N, int PL) {
    StageDesc d{};
    const int S = dstk::ct_nstages(N, PL);
    for (int s = 0; s < S; ++s) {
        d.ns[d.n] = dstk::ct_stage_ns(N, s, PL);
        d.r[d.n] = dstk::ct_radix(N, s, PL);
        d.off[d.n] = dstk::ct_tw_off(N, s, PL);
        if (d.ns[d.n] > 1) ++d.n;
    }
    return d;
}

// Table block of dst_table_doubles(N) = 6N doubles:
//   FP64: cos(π(t+1)/N) at [0, N), sin(πt/N) at [N, 2N), stage twiddles
//         exp(+2πi k r/(Ns R)) (complex) from 2N on (≤ N of them);
//   FP32 (from double 4N on, as floats): 4 sin²(π(t+1)/(2N)) at [0, N),
//         sin(πt/N) at [N, 2N), the twiddles (complex) from 2N on;
// each FP32 entry is the FP64 value rounded once.  The throughput plan's
// twiddles (when built) follow from double 6N on: FP64 (≤ N complex), then
// FP32 (≤ N complex).
__global__ void dst_twiddles_kernel(StageDesc d, int ntw, double2* W, float2* W32) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ntw; i += gridDim.x * blockDim.x) {
        int st = 0;
        while (st + 1 < d.n && i >= d.off[st + 1]) ++st;
        const int j = i - d.off[st];
        const int r = j / d.ns[st] + 1, k = j % d.ns[st];
        double sn, cs;
        sincospi(2.0 * (double)(k * r) / (double)(d.ns[st] * d.r[st]), &sn, &cs);
        W[i] = make_double2(cs, sn);
        W32[i] = make_float2((float)cs, (float)sn);
    }
}

__global__ void dst_tables_kernel(int N, double* base) {
    double* c = base;
    double* s = base + N;
    float* a32 = reinterpret_cast<float*>(base + 4 * N);
    float* s32 = a32 + N;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < N; t += gridDim.x * blockDim.x) {
        s[t] = sinpi((double)t / (double)N);
        s32[t] = (float)s[t];
        // evaluated as the reference forms the Laplacian eigenvalues:
        // cos.(π*(1:(n-1))/n) (laplacian.jl:17)
        c[t] = (t < N - 1) ? cos(M_PI * (double)(t + 1) / (double)N) : 0.0;
        const double h = sinpi((double)(t + 1) / (2.0 * (double)N));
        a32[t] = (t < N - 1) ? (float)(4.0 * h * h) : 0.0f;
    }
}

static cudaError_t twiddles_build(int N, int PL, double2* W, float2* W32, cudaStream_t st) {
    const int ntw = dstk::ct_tw_count(N, PL);
    if (ntw > N) return cudaErrorInvalidValue;  // the block holds at most N per plan
    if (ntw > 0) dst_twiddles_kernel<<<(ntw + 255) / 256, 256, 0, st>>>(stage_desc(N, PL), ntw, W, W32);
    return cudaGetLastError();
}

cudaError_t dst_tables_build(int N, double* base, cudaStream_t st) {
    dst_tables_kernel<<<(N + 255) / 256, 256, 0, st>>>(N, base);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    return twiddles_build(N, 0, reinterpret_cast<double2*>(base + 2 * N),
                          reinterpret_cast<float2*>(reinterpret_cast<float*>(base + 4 * N) + 2 * N), st);
}

DstPlan dst_plan_at(double* base, int N) {
    DstPlan p;
    p.N = N;
    p.c = base;
    p.s = base + N;
    p.W = reinterpret_cast<double2*>(base + 2 * N);
    p.a32 = reinterpret_cast<float*>(base + 4 * N);
    p.s32 = p.a32 + N;
    p.W32 = reinterpret_cast<float2*>(p.a32 + 2 * N);
    p.Wt = nullptr;
    p.Wt32 = nullptr;
    p.plan1 = p.planN = DST_PLAN_LATENCY;
    p.sims = 0;
    return p;
}

int dst_plan_create(DstPlan* p, int N, cudaStream_t st) {
    p->N = N;
    p->W = nullptr; p->s = nullptr; p->c = nullptr;
    if (!dst_supported(N)) return -1;
    double* base = nullptr;
    if (cudaMalloc(&base, sizeof(double) * dst_table_doubles_all(N)) != cudaSuccess) return -2;
    *p = dst_plan_at(base, N);
    if (dst_tables_build(N, base, st) != cudaSuccess) return -2;
    p->Wt = reinterpret_cast<double2*>(base + 6 * N);
    p->Wt32 = reinterpret_cast<float2*>(base + 8 * N);
    if (twiddles_build(N, dstk::ct_plan(N, 1), p->Wt, p->Wt32, st) != cudaSuccess) return -2;
    p->planN = DST_PLAN_AUTO;
    if (dst_init_attributes(N) != cudaSuccess) return -2;
    return 0;
}

void dst_plan_destroy(DstPlan* p) {
    if (p->c) cudaFree(p->c);  // the block starts at c
    p->W = nullptr; p->s = nullptr; p->c = nullptr;
    p->W32 = nullptr; p->s32 = nullptr; p->a32 = nullptr;
    p->Wt = nullptr; p->Wt32 = nullptr;
}

// Opt the kernels of length N into large dynamic shared memory (before any
// launch or graph capture).
cudaError_t dst_init_attributes(int N) {
    switch (N) {
#define IBPM_CASE(L) case L: return dst_attr_##L();
        IBPM_DST_LENGTHS(IBPM_CASE)
#undef IBPM_CASE
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_dst_x(const Geom& g, const DstPlan& px, const XPassArgs& a, cudaStream_t st) {
    switch (px.N) {
#define IBPM_CASE(L) case L: return dst_x_##L(g, px, a, st);
        IBPM_DST_LENGTHS(IBPM_CASE)
#undef IBPM_CASE
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_dst_y(const Geom& g, const DstPlan& py, const DstPlan& px, void* data, SlabMap map, int nslabs,
                         const SpecParams& sp, cudaStream_t st) {
    if (nslabs <= 0) return cudaSuccess;
    switch (py.N) {
#define IBPM_CASE(L) case L: return dst_y_##L(g, py, px, data, map, nslabs, sp, st);
        IBPM_DST_LENGTHS(IBPM_CASE)
#undef IBPM_CASE
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_dst_ybc(const Geom& g, const DstPlan& py, const DstPlan& px, void* out, SlabMap map, int nslabs,
                           const SpecParams& sp, const BtSynth& bs, cudaStream_t st) {
    if (nslabs <= 0) return cudaSuccess;
    switch (py.N) {
#define IBPM_CASE(L) case L: return dst_ybc_##L(g, py, px, out, map, nslabs, sp, bs, st);
        IBPM_DST_LENGTHS(IBPM_CASE)
#undef IBPM_CASE
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_dst_lines(const Geom& g, const DstPlan& px, const void* Y, SlabMap map, int nslabs,
                             void* samples, int f32, cudaStream_t st) {
    if (nslabs <= 0) return cudaSuccess;
    switch (px.N) {
#define IBPM_CASE(L) case L: return dst_lines_##L(g, px, Y, map, nslabs, samples, f32, st);
        IBPM_DST_LENGTHS(IBPM_CASE)
#undef IBPM_CASE
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace ibpm
