// Inverse-Laplacian solve that allocates no device memory.
//
// Some callers cannot call cudaMalloc: hosts whose device memory is owned by a
// pool or arena they do not share (a Julia or Python runtime with its own
// caching allocator, a solver embedded in a larger application with a fixed
// memory budget), or code that must run with no allocation at all once it is
// set up.  ibpm_lap_inv_noalloc serves them: the caller passes the right-hand
// side and the result buffer; the one intermediate slab of the solve and the
// transform tables live in file-scope __device__ arrays of fixed size, which
// every GPU that loads the library holds until the process exits
// (2.1 MB + 104 KB).
#include "../../include/ibpm_gpu.h"
#include "ibpm_internal.cuh"

#include <mutex>
#include <string>

using namespace ibpm;

namespace {

constexpr int kMaxN = 512;                                         // nx, ny <= 512
constexpr size_t kSlabDoubles = (size_t)(kMaxN - 1) * kMaxN;       // (ny-1) rows of pitch nx
// The supported lengths, each with a fixed block of 6N doubles (FP64 and
// FP32 tables of one length) at a fixed offset: 6 * 2168 doubles in all.
constexpr int kLengths[] = {32, 64, 128, 192, 200, 256, 384, 400, 512};
constexpr int kNumLengths = sizeof(kLengths) / sizeof(kLengths[0]);
constexpr size_t table_offset(int k) { return k == 0 ? 0 : table_offset(k - 1) + 6 * (size_t)kLengths[k - 1]; }
constexpr size_t kTableDoubles = table_offset(kNumLengths);

__device__ __align__(256) double g_noalloc_slab[kSlabDoubles];
__device__ __align__(256) double g_noalloc_tables[kTableDoubles];

struct DeviceScratch {
    bool ready = false;
    double* slab = nullptr;    // device address of g_noalloc_slab on this device
    double* tables = nullptr;  // device address of g_noalloc_tables on this device
};
constexpr int kMaxDevices = 64;
std::mutex g_mutex;
DeviceScratch g_scratch[kMaxDevices];

int length_index(int N) {
    for (int k = 0; k < kNumLengths; ++k)
        if (kLengths[k] == N) return k;
    return -1;
}

int noalloc_fail(int code, const std::string& msg) {
    set_global_error(msg.c_str());
    return code;
}

}  // namespace

extern "C" int ibpm_lap_inv_noalloc(int32_t nx, int32_t ny, const double* rhs, double* x, void* stream) {
    if (!rhs || !x) return noalloc_fail(IBPM_ERR_INVALID, "ibpm_lap_inv_noalloc: null buffer");
    if (nx > kMaxN || ny > kMaxN)
        return noalloc_fail(IBPM_ERR_INVALID, "ibpm_lap_inv_noalloc: nx and ny must be at most 512 (got " +
                                                  std::to_string(nx) + " x " + std::to_string(ny) + ")");
    if (length_index(nx) < 0 || length_index(ny) < 0)
        return noalloc_fail(IBPM_ERR_UNSUPPORTED,
                            "ibpm_lap_inv_noalloc: nx and ny must be one of 32, 64, 128, 192, 200, 256, 384, "
                            "400, 512");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return noalloc_fail(IBPM_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return noalloc_fail(IBPM_ERR_INVALID, "device ordinal out of range");

    std::lock_guard<std::mutex> lock(g_mutex);
    DeviceScratch& ds = g_scratch[dev];
    if (!ds.ready) {
        // Once per device, with that device current: the host-side names of
        // the __device__ arrays are not device addresses, so ask the runtime.
        e = cudaGetSymbolAddress(reinterpret_cast<void**>(&ds.slab), g_noalloc_slab);
        if (e != cudaSuccess)
            return noalloc_fail(IBPM_ERR_CUDA, std::string("cudaGetSymbolAddress(slab): ") + cudaGetErrorString(e));
        e = cudaGetSymbolAddress(reinterpret_cast<void**>(&ds.tables), g_noalloc_tables);
        if (e != cudaSuccess)
            return noalloc_fail(IBPM_ERR_CUDA, std::string("cudaGetSymbolAddress(tables): ") + cudaGetErrorString(e));
        // Every supported length's tables, once: later calls (and a graph
        // that captured one) find them in place, whatever sizes ran between.
        for (int k = 0; k < kNumLengths; ++k) {
            e = dst_init_attributes(kLengths[k]);
            if (e == cudaSuccess) e = dst_tables_build(kLengths[k], ds.tables + table_offset(k), st);
            if (e != cudaSuccess)
                return noalloc_fail(IBPM_ERR_CUDA, std::string("set-up: ") + cudaGetErrorString(e));
        }
        ds.ready = true;
    }
    double* tx = ds.tables + table_offset(length_index(nx));
    double* ty = ds.tables + table_offset(length_index(ny));
    const Geom g = make_geom(nx, ny, 1);
    const DstPlan px = dst_plan_at(tx, nx), py = dst_plan_at(ty, ny);
    // Every slab element that the transforms read (columns < nx-1) is written
    // by this copy, so nothing left by an earlier call is read.
    const size_t row = sizeof(double) * g.n1;
    e = cudaMemcpy2DAsync(ds.slab, sizeof(double) * g.P, rhs, row, row, g.n2, cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return noalloc_fail(IBPM_ERR_CUDA, std::string("copy in: ") + cudaGetErrorString(e));
    SlabMap m;
    m.nlev = 1; m.lev0 = 0; m.lstride = g.S; m.bstride = g.S;
    XPassArgs a{};
    a.in = ds.slab; a.out = ds.slab; a.in_map = m; a.out_map = m;
    a.nslabs = 1; a.line0 = 0; a.line1 = g.n2; a.load = XLOAD_PLAIN; a.emit = XEMIT_STORE;
    SpecParams sp{};
    sp.mode = SPEC_DELTA;
    sp.scale = 1.0 / (4.0 * nx * ny);  // get_lap_inv, laplacian.jl:38
    if ((e = launch_dst_x(g, px, a, st)) != cudaSuccess ||
        (e = launch_dst_y(g, py, px, ds.slab, m, 1, sp, st)) != cudaSuccess ||
        (e = launch_dst_x(g, px, a, st)) != cudaSuccess)
        return noalloc_fail(IBPM_ERR_CUDA, std::string("solve: ") + cudaGetErrorString(e));
    e = cudaMemcpy2DAsync(x, row, ds.slab, sizeof(double) * g.P, row, g.n2, cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return noalloc_fail(IBPM_ERR_CUDA, std::string("copy out: ") + cudaGetErrorString(e));
    return IBPM_OK;
}
