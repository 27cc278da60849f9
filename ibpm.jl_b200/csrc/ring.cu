// Dispatch and tables of the spectral level chain (kernels: ring_kernels.cuh,
// one instantiation unit per grid shape: ring_<nx>_<ny>.cu).
#include "ibpm_internal.cuh"

#include <math.h>

namespace ibpm {

cudaError_t ring_32_32(const Geom&, const DstPlan&, const DstPlan&, const RingArgs&, int, cudaStream_t);
cudaError_t ring_attr_32_32();
cudaError_t ring_64_64(const Geom&, const DstPlan&, const DstPlan&, const RingArgs&, int, cudaStream_t);
cudaError_t ring_attr_64_64();
cudaError_t ring_128_128(const Geom&, const DstPlan&, const DstPlan&, const RingArgs&, int, cudaStream_t);
cudaError_t ring_attr_128_128();
cudaError_t ring_192_192(const Geom&, const DstPlan&, const DstPlan&, const RingArgs&, int, cudaStream_t);
cudaError_t ring_attr_192_192();
cudaError_t ring_200_200(const Geom&, const DstPlan&, const DstPlan&, const RingArgs&, int, cudaStream_t);
cudaError_t ring_attr_200_200();
cudaError_t ring_256_256(const Geom&, const DstPlan&, const DstPlan&, const RingArgs&, int, cudaStream_t);
cudaError_t ring_attr_256_256();
cudaError_t ring_384_384(const Geom&, const DstPlan&, const DstPlan&, const RingArgs&, int, cudaStream_t);
cudaError_t ring_attr_384_384();
cudaError_t ring_400_400(const Geom&, const DstPlan&, const DstPlan&, const RingArgs&, int, cudaStream_t);
cudaError_t ring_attr_400_400();
cudaError_t ring_512_512(const Geom&, const DstPlan&, const DstPlan&, const RingArgs&, int, cudaStream_t);
cudaError_t ring_attr_512_512();
cudaError_t ring_768_768(const Geom&, const DstPlan&, const DstPlan&, const RingArgs&, int, cudaStream_t);
cudaError_t ring_attr_768_768();
cudaError_t ring_1024_1024(const Geom&, const DstPlan&, const DstPlan&, const RingArgs&, int, cudaStream_t);
cudaError_t ring_attr_1024_1024();
cudaError_t ring_64_32(const Geom&, const DstPlan&, const DstPlan&, const RingArgs&, int, cudaStream_t);
cudaError_t ring_attr_64_32();
cudaError_t ring_128_64(const Geom&, const DstPlan&, const DstPlan&, const RingArgs&, int, cudaStream_t);
cudaError_t ring_attr_128_64();
cudaError_t ring_400_200(const Geom&, const DstPlan&, const DstPlan&, const RingArgs&, int, cudaStream_t);
cudaError_t ring_attr_400_200();

bool ring_supported(int nx, int ny) {
    switch (nx * 10000 + ny) {
        case 320032: return true;
        case 640064: return true;
        case 1280128: return true;
        case 1920192: return true;
        case 2000200: return true;
        case 2560256: return true;
        case 3840384: return true;
        case 4000400: return true;
        case 5120512: return true;
        case 7680768: return true;
        case 10241024: return true;
        case 640032: return true;
        case 1280064: return true;
        case 4000200: return true;
        default: return false;
    }
}

cudaError_t ring_init_attributes(int nx, int ny) {
    switch (nx * 10000 + ny) {
        case 320032: return ring_attr_32_32();
        case 640064: return ring_attr_64_64();
        case 1280128: return ring_attr_128_128();
        case 1920192: return ring_attr_192_192();
        case 2000200: return ring_attr_200_200();
        case 2560256: return ring_attr_256_256();
        case 3840384: return ring_attr_384_384();
        case 4000400: return ring_attr_400_400();
        case 5120512: return ring_attr_512_512();
        case 7680768: return ring_attr_768_768();
        case 10241024: return ring_attr_1024_1024();
        case 640032: return ring_attr_64_32();
        case 1280064: return ring_attr_128_64();
        case 4000200: return ring_attr_400_200();
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_ring(const Geom& g, const DstPlan& px, const DstPlan& py, const RingArgs& a, int nbatch,
                        cudaStream_t st) {
    switch (g.nx * 10000 + g.ny) {
        case 320032: return ring_32_32(g, px, py, a, nbatch, st);
        case 640064: return ring_64_64(g, px, py, a, nbatch, st);
        case 1280128: return ring_128_128(g, px, py, a, nbatch, st);
        case 1920192: return ring_192_192(g, px, py, a, nbatch, st);
        case 2000200: return ring_200_200(g, px, py, a, nbatch, st);
        case 2560256: return ring_256_256(g, px, py, a, nbatch, st);
        case 3840384: return ring_384_384(g, px, py, a, nbatch, st);
        case 4000400: return ring_400_400(g, px, py, a, nbatch, st);
        case 5120512: return ring_512_512(g, px, py, a, nbatch, st);
        case 7680768: return ring_768_768(g, px, py, a, nbatch, st);
        case 10241024: return ring_1024_1024(g, px, py, a, nbatch, st);
        case 640032: return ring_64_32(g, px, py, a, nbatch, st);
        case 1280064: return ring_128_64(g, px, py, a, nbatch, st);
        case 4000200: return ring_400_200(g, px, py, a, nbatch, st);
        default: return cudaErrorInvalidValue;
    }
}

int ring_nbands(const Geom& g) { return 1; }

// 2 sin(π a b / N) with the product reduced modulo 2N (exact argument).
__device__ __forceinline__ double sine2(long long a, long long b, int N) {
    return 2.0 * sinpi((double)((a * b) % (2LL * N)) / (double)N);
}

__global__ void ring_tables_kernel(int nx, int ny, int len, double* base) {
    double* sxl = base;
    double* sxr = base + len;
    double* syb = base + 2 * len;
    double* syt = base + 3 * len;
    double* sx0 = base + 4 * len;
    double* sxN = base + 5 * len;
    double* sy0 = base + 6 * len;
    double* syN = base + 7 * len;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < len; t += gridDim.x * blockDim.x) {
        if (t < nx - 1) {
            sxl[t] = sine2(nx / 4, t + 1, nx);
            sxr[t] = sine2(3 * nx / 4, t + 1, nx);
            sx0[t] = sine2(1, t + 1, nx);
            sxN[t] = sine2(nx - 1, t + 1, nx);
        }
        if (t < ny - 1) {
            syb[t] = sine2(ny / 4, t + 1, ny);
            syt[t] = sine2(3 * ny / 4, t + 1, ny);
            sy0[t] = sine2(1, t + 1, ny);
            syN[t] = sine2(ny - 1, t + 1, ny);
        }
    }
}

cudaError_t ring_tables_build(const Geom& g, int len, double* base, cudaStream_t st) {
    ring_tables_kernel<<<(len + 255) / 256, 256, 0, st>>>(g.nx, g.ny, len, base);
    return cudaGetLastError();
}

}  // namespace ibpm
