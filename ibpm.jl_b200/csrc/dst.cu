// Transform tables and length dispatch of the batched DST-I kernels
// (kernels: dst_kernels.cuh, one instantiation unit per length: dst_n<N>.cu).
#include "ibpm_internal.cuh"

#include <math.h>

namespace ibpm {

cudaError_t dst_x_32(const Geom&, const DstPlan&, const XPassArgs&, cudaStream_t);
cudaError_t dst_y_32(const Geom&, const DstPlan&, const DstPlan&, double*, SlabMap, int, const SpecParams&, cudaStream_t);
cudaError_t dst_attr_32();
cudaError_t dst_x_64(const Geom&, const DstPlan&, const XPassArgs&, cudaStream_t);
cudaError_t dst_y_64(const Geom&, const DstPlan&, const DstPlan&, double*, SlabMap, int, const SpecParams&, cudaStream_t);
cudaError_t dst_attr_64();
cudaError_t dst_x_128(const Geom&, const DstPlan&, const XPassArgs&, cudaStream_t);
cudaError_t dst_y_128(const Geom&, const DstPlan&, const DstPlan&, double*, SlabMap, int, const SpecParams&, cudaStream_t);
cudaError_t dst_attr_128();
cudaError_t dst_x_192(const Geom&, const DstPlan&, const XPassArgs&, cudaStream_t);
cudaError_t dst_y_192(const Geom&, const DstPlan&, const DstPlan&, double*, SlabMap, int, const SpecParams&, cudaStream_t);
cudaError_t dst_attr_192();
cudaError_t dst_x_200(const Geom&, const DstPlan&, const XPassArgs&, cudaStream_t);
cudaError_t dst_y_200(const Geom&, const DstPlan&, const DstPlan&, double*, SlabMap, int, const SpecParams&, cudaStream_t);
cudaError_t dst_attr_200();
cudaError_t dst_x_256(const Geom&, const DstPlan&, const XPassArgs&, cudaStream_t);
cudaError_t dst_y_256(const Geom&, const DstPlan&, const DstPlan&, double*, SlabMap, int, const SpecParams&, cudaStream_t);
cudaError_t dst_attr_256();
cudaError_t dst_x_384(const Geom&, const DstPlan&, const XPassArgs&, cudaStream_t);
cudaError_t dst_y_384(const Geom&, const DstPlan&, const DstPlan&, double*, SlabMap, int, const SpecParams&, cudaStream_t);
cudaError_t dst_attr_384();
cudaError_t dst_x_400(const Geom&, const DstPlan&, const XPassArgs&, cudaStream_t);
cudaError_t dst_y_400(const Geom&, const DstPlan&, const DstPlan&, double*, SlabMap, int, const SpecParams&, cudaStream_t);
cudaError_t dst_attr_400();
cudaError_t dst_x_512(const Geom&, const DstPlan&, const XPassArgs&, cudaStream_t);
cudaError_t dst_y_512(const Geom&, const DstPlan&, const DstPlan&, double*, SlabMap, int, const SpecParams&, cudaStream_t);
cudaError_t dst_attr_512();
cudaError_t dst_x_768(const Geom&, const DstPlan&, const XPassArgs&, cudaStream_t);
cudaError_t dst_y_768(const Geom&, const DstPlan&, const DstPlan&, double*, SlabMap, int, const SpecParams&, cudaStream_t);
cudaError_t dst_attr_768();
cudaError_t dst_x_1024(const Geom&, const DstPlan&, const XPassArgs&, cudaStream_t);
cudaError_t dst_y_1024(const Geom&, const DstPlan&, const DstPlan&, double*, SlabMap, int, const SpecParams&, cudaStream_t);
cudaError_t dst_attr_1024();
cudaError_t dst_x_2048(const Geom&, const DstPlan&, const XPassArgs&, cudaStream_t);
cudaError_t dst_y_2048(const Geom&, const DstPlan&, const DstPlan&, double*, SlabMap, int, const SpecParams&, cudaStream_t);
cudaError_t dst_attr_2048();

// Supported transform lengths N = nx or ny: 32, 64, 128, 192, 200, 256, 384, 400, 512, 768, 1024, 2048.
bool dst_supported(int N) {
    switch (N) {
        case 32:
        case 64:
        case 128:
        case 192:
        case 200:
        case 256:
        case 384:
        case 400:
        case 512:
        case 768:
        case 1024:
        case 2048:
            return true;
        default:
            return false;
    }
}

__global__ void dst_tables_kernel(int N, double2* W, double* s, double* c) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < N; t += gridDim.x * blockDim.x) {
        double sn, cs;
        sincospi(2.0 * (double)t / (double)N, &sn, &cs);
        W[t] = make_double2(cs, sn);            // exp(+2πi t/N)
        s[t] = sinpi((double)t / (double)N);    // sin(π t/N)
        // cos(π (t+1)/N), evaluated as the reference forms the Laplacian
        // eigenvalues: cos.(π*(1:(n-1))/n) (laplacian.jl:173)
        if (t < N - 1) c[t] = cos(M_PI * (double)(t + 1) / (double)N);
    }
}

int dst_plan_create(DstPlan* p, int N, cudaStream_t st) {
    p->N = N;
    p->W = nullptr; p->s = nullptr; p->c = nullptr;
    if (!dst_supported(N)) return -1;
    if (cudaMalloc(&p->W, sizeof(double2) * N) != cudaSuccess) return -2;
    if (cudaMalloc(&p->s, sizeof(double) * N) != cudaSuccess) return -2;
    if (cudaMalloc(&p->c, sizeof(double) * N) != cudaSuccess) return -2;
    dst_tables_kernel<<<(N + 255) / 256, 256, 0, st>>>(N, p->W, p->s, p->c);
    if (cudaGetLastError() != cudaSuccess) return -2;
    if (dst_init_attributes(N) != cudaSuccess) return -2;
    return 0;
}

cudaError_t dst_tables_build(int N, double2* W, double* s, double* c, cudaStream_t st) {
    dst_tables_kernel<<<(N + 255) / 256, 256, 0, st>>>(N, W, s, c);
    return cudaGetLastError();
}

void dst_plan_destroy(DstPlan* p) {
    if (p->W) cudaFree(p->W);
    if (p->s) cudaFree(p->s);
    if (p->c) cudaFree(p->c);
    p->W = nullptr; p->s = nullptr; p->c = nullptr;
}

// Opt the kernels of length N into large dynamic shared memory (before any
// launch or graph capture).
cudaError_t dst_init_attributes(int N) {
    switch (N) {
        case 32: return dst_attr_32();
        case 64: return dst_attr_64();
        case 128: return dst_attr_128();
        case 192: return dst_attr_192();
        case 200: return dst_attr_200();
        case 256: return dst_attr_256();
        case 384: return dst_attr_384();
        case 400: return dst_attr_400();
        case 512: return dst_attr_512();
        case 768: return dst_attr_768();
        case 1024: return dst_attr_1024();
        case 2048: return dst_attr_2048();
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_dst_x(const Geom& g, const DstPlan& px, const XPassArgs& a, cudaStream_t st) {
    switch (px.N) {
        case 32: return dst_x_32(g, px, a, st);
        case 64: return dst_x_64(g, px, a, st);
        case 128: return dst_x_128(g, px, a, st);
        case 192: return dst_x_192(g, px, a, st);
        case 200: return dst_x_200(g, px, a, st);
        case 256: return dst_x_256(g, px, a, st);
        case 384: return dst_x_384(g, px, a, st);
        case 400: return dst_x_400(g, px, a, st);
        case 512: return dst_x_512(g, px, a, st);
        case 768: return dst_x_768(g, px, a, st);
        case 1024: return dst_x_1024(g, px, a, st);
        case 2048: return dst_x_2048(g, px, a, st);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_dst_y_solve(const Geom& g, const DstPlan& py, const DstPlan& px, double* data, SlabMap map,
                               int nslabs, const SpecParams& sp, cudaStream_t st) {
    if (nslabs <= 0) return cudaSuccess;
    switch (py.N) {
        case 32: return dst_y_32(g, py, px, data, map, nslabs, sp, st);
        case 64: return dst_y_64(g, py, px, data, map, nslabs, sp, st);
        case 128: return dst_y_128(g, py, px, data, map, nslabs, sp, st);
        case 192: return dst_y_192(g, py, px, data, map, nslabs, sp, st);
        case 200: return dst_y_200(g, py, px, data, map, nslabs, sp, st);
        case 256: return dst_y_256(g, py, px, data, map, nslabs, sp, st);
        case 384: return dst_y_384(g, py, px, data, map, nslabs, sp, st);
        case 400: return dst_y_400(g, py, px, data, map, nslabs, sp, st);
        case 512: return dst_y_512(g, py, px, data, map, nslabs, sp, st);
        case 768: return dst_y_768(g, py, px, data, map, nslabs, sp, st);
        case 1024: return dst_y_1024(g, py, px, data, map, nslabs, sp, st);
        case 2048: return dst_y_2048(g, py, px, data, map, nslabs, sp, st);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace ibpm
