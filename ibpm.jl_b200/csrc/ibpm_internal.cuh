// Internal definitions shared by the kernels and the C ABI of libibpm_gpu.so.
//
// Device layout (all FP64):
//   * A Γ-like field (Γ, ψ, nonlinear term, right-hand sides) of one level is a
//     "slab" of (ny-1) rows of pitch P = nx doubles; element (i, j) (0-based,
//     i < nx-1 fastest, j < ny-1) sits at row j, column i.  The reference keeps
//     the same field as a column-major (nx-1)×(ny-1) matrix
//     (src/fluid-domain/fluid-domain.jl:55); the pitch pads each row to 32 B.
//   * A field with levels (and optionally a batch of right-hand sides) is
//     slab-major: slab index = batch * mg + level.
//   * A flux field of one level is the reference's flat vector of nq doubles:
//     qx (nx+1)×ny column-major, then qy nx×(ny+1) (fluid-domain.jl:64-65).
//   * Boundary vectors (Γbc / ψbc) use the reference's segment offsets
//     LEFT = 0, RIGHT = ny+1, BOT = 2(ny+1), TOP = 2(ny+1)+nx+1
//     (fluid-domain.jl:68-69); element v of a segment belongs to the edge
//     vertex v (0 … nx or 0 … ny).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

namespace ibpm {

struct Geom {
    int nx, ny, mg;
    int n1, n2;          // nx-1, ny-1
    int P;               // slab pitch (doubles) = nx
    long long S;         // slab size (doubles) = P * n2
    int nu, nv, nq;      // flux sizes
    int L, R, B, T, nbc; // boundary vector offsets and length
};

inline Geom make_geom(int nx, int ny, int mg) {
    Geom g;
    g.nx = nx; g.ny = ny; g.mg = mg;
    g.n1 = nx - 1; g.n2 = ny - 1;
    g.P = nx;
    g.S = (long long)g.P * g.n2;
    g.nu = ny * (nx + 1);
    g.nv = nx * (ny + 1);
    g.nq = g.nu + g.nv;
    g.L = 0; g.R = ny + 1; g.B = 2 * (ny + 1); g.T = 2 * (ny + 1) + nx + 1;
    g.nbc = 2 * (nx + 1) + 2 * (ny + 1);
    return g;
}

// Maps blockIdx.y (or any flat slab counter) to (batch, level) and offsets.
struct SlabMap {
    int nlev;            // levels per batch member handled by the launch
    int lev0;            // first level
    long long bstride;   // doubles between batch members
    long long lstride;   // doubles between levels
    __host__ __device__ int level(int y) const { return lev0 + y % nlev; }
    __host__ __device__ int batch(int y) const { return y / nlev; }
    __host__ __device__ long long off(int y) const {
        return (long long)(y / nlev) * bstride + (long long)(lev0 + y % nlev) * lstride;
    }
};

// Edge value of get_bc! (src/fluid-operators/mg-utils.jl:7-32) for vertex v of
// one segment, read from the coarser level's slab `rc`.  Along the segment the
// coarse samples start at coarse index c0 (x for BOT/TOP, y for LEFT/RIGHT)
// and sit at fixed cross index cfix: even v copies coarse point c0 + v/2, odd v
// averages the two coarse points around it.
//   BOT: c0 = nx/4-1 along x, cfix = ny/4-1      TOP: same, cfix = 3ny/4-1
//   LEFT: c0 = ny/4-1 along y, cfix = nx/4-1     RIGHT: same, cfix = 3nx/4-1
__device__ __forceinline__ double getbc_x(const double* __restrict__ rc, int P, int v,
                                          int c0, int jfix) {
    if ((v & 1) == 0) return rc[(long long)jfix * P + c0 + (v >> 1)];
    int ia = c0 + ((v + 1) >> 1);
    return 0.5 * (rc[(long long)jfix * P + ia] + rc[(long long)jfix * P + ia - 1]);
}
__device__ __forceinline__ double getbc_y(const double* __restrict__ rc, int P, int v,
                                          int c0, int ifix) {
    if ((v & 1) == 0) return rc[(long long)(c0 + (v >> 1)) * P + ifix];
    int ja = c0 + ((v + 1) >> 1);
    return 0.5 * (rc[(long long)ja * P + ifix] + rc[(long long)(ja - 1) * P + ifix]);
}

// The four edges of a fine level's boundary, sampled from the coarser slab.
struct CoarseBC {
    const double* rc;    // coarser-level slab, or nullptr for zero BCs
    int P, nx, ny;
    __device__ __forceinline__ double bot(int v) const {
        return rc ? getbc_x(rc, P, v, nx / 4 - 1, ny / 4 - 1) : 0.0;
    }
    __device__ __forceinline__ double top(int v) const {
        return rc ? getbc_x(rc, P, v, nx / 4 - 1, 3 * ny / 4 - 1) : 0.0;
    }
    __device__ __forceinline__ double left(int v) const {
        return rc ? getbc_y(rc, P, v, ny / 4 - 1, nx / 4 - 1) : 0.0;
    }
    __device__ __forceinline__ double right(int v) const {
        return rc ? getbc_y(rc, P, v, ny / 4 - 1, 3 * nx / 4 - 1) : 0.0;
    }
};

// ---------------------------------------------------------------------------
// Programmatic dependent launch: every kernel of the step is launched with
// cudaLaunchAttributeProgrammaticStreamSerialization, so it can be scheduled
// while its predecessor drains.  A kernel may stage constant tables first, but
// must call pdl_wait() before touching anything an earlier kernel wrote;
// pdl_trigger() lets the next kernel launch.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// Asynchronous global → shared copies (cp.async): all of a thread's copies
// are in flight together; cp_async_wait() + a barrier makes them visible.
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(s), "l"(gmem) : "memory");
}
template <int B> __device__ __forceinline__ void cp_async(void* smem, const void* gmem) {
    static_assert(B == 4 || B == 8 || B == 16, "cp.async copies 4, 8 or 16 bytes");
    if constexpr (B == 4) cp_async4(smem, gmem);
    else if constexpr (B == 8) cp_async8(smem, gmem);
    else cp_async16(smem, gmem);
}
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_all;" ::: "memory"); }

bool pdl_enabled();

// 1/d by Newton–Raphson: a single-precision seed (relative error ≤ 2^-23),
// refined twice with r ← r + r(1 − d r), which squares the error each time
// (2^-46, then below the double rounding).  Within 1-2 ulp of 1/d, with no
// branches; used where a full IEEE division per element would dominate.
__device__ __forceinline__ double nr_rcp(double d) {
    double r = (double)__frcp_rn((float)d);
    double e = fma(-d, r, 1.0);
    r = fma(r, e, r);
    e = fma(-d, r, 1.0);
    return fma(r, e, r);
}

template <typename... KArgs, typename... Args>
cudaError_t launch_k(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                     Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = pdl_enabled() ? 1 : 0;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}

// ---------------------------------------------------------------------------
// Host-side launchers (defined in the .cu files).
// ---------------------------------------------------------------------------
struct DstPlan {
    int N;               // transform length nx (x-pass) or ny (y-pass) = n + 1
    double2* W;          // device: per-stage FFT twiddles (stage-contiguous, ≤ N entries)
    double* s;           // device: sin(π m/N), m < N
    double* c;           // device: cos(π (k+1)/N), k < N-1 (Laplacian eigenvalues)
    // the same tables rounded to FP32, for the FP32 transforms
    float2* W32;
    float* s32;
    float* a32;          // 2 (1 − cos(π (k+1)/N)) = 4 sin²(π (k+1)/(2N)), free of cancellation
    // stage twiddles of the throughput plan (radix 8), FP64 and FP32; null
    // when the block holds only the latency plan's tables
    double2* Wt;
    float2* Wt32;
    // plan of single-slab and of multi-slab launches (DST_PLAN_*)
    int plan1, planN;
    // simulations sharing each launch (batch groups; 0 or 1: one): the plan
    // follows the slabs of one simulation, so a member computes what it
    // computes alone
    int sims;
};
// DST_PLAN_AUTO (multi-slab launches only): the throughput plan for launches
// of at least kAutoWideSlabs slabs (the columns of B, the moving bodies'
// unit solves), else the single-slab plan (the levels of one step).
enum DstPlanKind { DST_PLAN_LATENCY = 0, DST_PLAN_THROUGHPUT = 1, DST_PLAN_AUTO = 2 };
constexpr int kAutoWideSlabs = 4;
// Doubles in the table block of one length (FP64 tables, then FP32 tables),
// and with the throughput plan's twiddles after them.
inline long long dst_table_doubles(int N) { return 6LL * N; }
inline long long dst_table_doubles_all(int N) { return 9LL * N; }

bool dst_supported(int N);
int dst_plan_create(DstPlan* p, int N, cudaStream_t st);  // 0 on success
cudaError_t dst_init_attributes(int N);
// Fill the table block of length N (dst_table_doubles(N) doubles) in
// caller-provided device memory and view it as a plan.
cudaError_t dst_tables_build(int N, double* base, cudaStream_t st);
DstPlan dst_plan_at(double* base, int N);
// Error text returned by ibpm_last_error(NULL).
void set_global_error(const char* msg);
void dst_plan_destroy(DstPlan* p);

// Spectral divisor applied between the two y-transforms of a Poisson solve:
//   DELTA: w ← (w / Λ) · scale                       (Δ⁻¹, laplacian.jl:24-41)
//   AINV:  w ← (w / (1 + Λ·dt / den[lev])) · scale    (A⁻¹, laplacian.jl:61-71)
enum SpecMode { SPEC_DELTA = 0, SPEC_AINV = 1 };
struct SpecParams {
    int mode;
    int f32;             // data and transforms in FP32 (the refinement correction)
    double scale;        // 1 / (4 nx ny)
    double dt;
    double den[8];       // 2 Re hc² per level
    // a launch over the slabs of several simulations of one grid (batch
    // groups): per simulation (the slab map's batch index) den[0..7] then dt,
    // 9 doubles each, in place of den and dt; nullptr otherwise
    const double* mden;
};

// x-direction DST-I of every line of the slabs selected by `map` over lines
// [line0, line1).  The load mode fixes how the input line is formed and the
// precision of the transform; the emit mode how the result is stored.
//   FP64 transforms (the reference's arithmetic):
//     XLOAD_PLAIN    b (double)
//     XLOAD_BC       b + apply_bc!(·, get_bc!(coarser), 1)            (mg-utils.jl:7-60)
//   FP32 transforms (the correction of one FP64-residual refinement sweep):
//     XLOAD_F32      b (float)
//     XLOAD_RES_LAP  Γ + apply_bc!(get_bc!(ψ coarser)) − L ψ̃   (double → float)
//     XLOAD_RES_A    b − (I + c L) x̃                            (double → float)
//   with L x = 4x − Σ neighbours (zero Dirichlet edges) the operator whose
//   inverse the DST-I solve with Λ applies, x̃ / ψ̃ the current solution (aux).
//     XEMIT_STORE    out = v (double)       XEMIT_SUB      out −= v (double)
//     XEMIT_F32      out = v (float)        XEMIT_ADD      out += v (double)
//     XEMIT_ADD_FROM out = aux + v          XEMIT_ACC_SUB  aux += v; out −= aux
//   and the last pass of a boundary-transfer vort2flux! (bt.cu), which
//   transforms the sum of the interior and edge parts of the x-spectrum:
//     XLOAD_SUM      in + in2 (double)     XLOAD_F32_SUM  in + in2 (float)
// The coarser-level field of XLOAD_BC / RES_LAP is read only for slabs whose
// level is below the coarsest (a multi-level launch includes the coarsest).
enum XLoad { XLOAD_PLAIN = 0, XLOAD_BC = 1, XLOAD_F32 = 2, XLOAD_RES_LAP = 3, XLOAD_RES_A = 4, XLOAD_SUM = 5,
             XLOAD_F32_SUM = 6 };
//     XEMIT_ADD_STORE out += v; aux = v (double; the adjoint level chain)
enum XEmit { XEMIT_STORE = 0, XEMIT_SUB = 1, XEMIT_F32 = 2, XEMIT_ADD = 3, XEMIT_ADD_FROM = 4, XEMIT_ACC_SUB = 5,
             XEMIT_ADD_STORE = 6 };
struct XPassArgs {
    const void* in; void* out;
    SlabMap in_map, out_map;
    const void* in2; SlabMap in2_map;            // XLOAD_SUM / F32_SUM: second addend
    const double* coarse;  SlabMap coarse_map;   // XLOAD_BC / RES_LAP: coarser-level field
    double* aux; SlabMap aux_map;                // RES_*: current solution; ADD_FROM / ACC_SUB (see above)
    double cA;                                   // XLOAD_RES_A: c = dt / (2 Re hc²)
    const double* mcA;                           // per simulation of a batch group (in_map's batch), or nullptr
    int nslabs, line0, line1;
    int load, emit;
};
cudaError_t launch_dst_x(const Geom& g, const DstPlan& px, const XPassArgs& a, cudaStream_t st);



// y-direction pass of a Poisson-type solve, in place on every slab selected by
// `map`: DST-I, spectral divide (SpecParams), DST-I.
cudaError_t launch_dst_y(const Geom& g, const DstPlan& py, const DstPlan& px_cos, void* data, SlabMap map,
                         int nslabs, const SpecParams& sp, cudaStream_t st);

// ---------------------------------------------------------------------------
// Boundary-transfer form of vort2flux! (bt.cu).  Δ⁻¹ is linear, so each
// level's streamfunction splits into an interior and an edge part,
//     ψ_ℓ = Δ⁻¹ Γ_ℓ + Δ⁻¹ apply_bc!(e_ℓ),   e_ℓ = get_bc!(ψ_{ℓ+1})
// (curl.jl:147-158, mg-utils.jl:7-60), and the edge vectors chain as
//     e_ℓ = get_bc!(Δ⁻¹ Γ_{ℓ+1}) + R e_{ℓ+1},   R = get_bc! ∘ Δ⁻¹ ∘ apply_bc!,
// R one nE×nE matrix for every level (the reference's Δ⁻¹ carries no h,
// models.jl:46).  An edge vector holds the nE = 2(nx−1) + 2(ny−1) entries that
// apply_bc! adds: bottom i = 1…nx−1, top, left j = 1…ny−1, right.
// The x-spectrum of apply_bc!(e) is known in closed form (one sine transform
// of the bottom and top rows, two sines for the left and right columns), so
// the edge part is one y-pass from e and the last x-pass adds both parts.
// Line samples of a level (what get_bc! reads from it): the row at ny/4 and
// at 3ny/4 (x = nx/4 … 3nx/4, nx/2+1 values each), then the column at nx/4 and
// at 3nx/4 (y = ny/4 … 3ny/4), each taken from the y-pass output (x-spectral).
// ---------------------------------------------------------------------------
inline int bt_edge_len(const Geom& g) { return 2 * g.n1 + 2 * g.n2; }
inline int bt_edge_pitch(const Geom& g) { return (bt_edge_len(g) + 3) & ~3; }  // R row pitch
inline int bt_sample_len(const Geom& g) { return g.nx + g.ny + 4; }
struct BtSynth {
    const double* e;      // edge vectors, level-major (bt_edge_pitch apart), FP64
    const double* sx;     // sin(π t/nx), t < nx, of the x-length (FP64)
    int nx;
};
cudaError_t launch_dst_ybc(const Geom& g, const DstPlan& py, const DstPlan& px, void* out, SlabMap map, int nslabs,
                           const SpecParams& sp, const BtSynth& bs, cudaStream_t st);
// The line samples (FP64) of the levels of `map` from Y (FP32 when f32).
cudaError_t launch_dst_lines(const Geom& g, const DstPlan& px, const void* Y, SlabMap map, int nslabs,
                             void* samples, int f32, cudaStream_t st);
// The chain in a rank-k basis of R (R ≈ Q W, Q orthonormal columns,
// W = Qᵀ R, k ≈ 135 for FP64 accuracy whatever the grid size: R is the
// Green's function between well-separated point sets, smooth, with fast
// decaying singular values):
//     p_ℓ = W g_ℓ (g_ℓ = get_bc!(samples of ℓ+1)),  ℓ = 0 … mg−2
//         (as Ws · samples, Ws = W with get_bc!'s averaging folded in)
//     e_ℓ = g_ℓ + Σ_{m=0}^{mg−3−ℓ} U_m p_{ℓ+1+m},   U_m = Q (W Q)^m
// which is e_ℓ = g_ℓ + R e_{ℓ+1} unrolled (two launches, none serial).
struct BtChainArgs {
    const double* W;        // Ws: k × sample pitch (bt_sample_len rounded to 4), row-major
    const double* U;        // mg−2 matrices nE × kp, row-major
    const double* samples;  // bt_sample_len per level, level-major
    double* p;              // (mg−1) × kp projections
    double* e;              // edge vectors, level-major, bt_edge_pitch apart
    int k, kp;              // rank and its pitch (multiple of 4)
    int nsim;               // simulations of one grid (batch groups; 0 means 1): samples, p
                            // and e of simulation s follow those of s−1 (mg·bt_sample_len,
                            // (mg−1)·kp and mg·bt_edge_pitch doubles apart)
};
cudaError_t launch_bt_project(const Geom& g, const BtChainArgs& a, cudaStream_t st);
cudaError_t launch_bt_expand(const Geom& g, const BtChainArgs& a, cudaStream_t st);
// Setup of R: unit sources of edge entries [c0, c0 + ncol) into ncol slabs
// (bstride apart, zeroed first), and the gather of their solves' get_bc!
// entries into R's columns (FP64).
cudaError_t launch_bt_unit_src(const Geom& g, int c0, int ncol, double* G, long long bstride, cudaStream_t st);
cudaError_t launch_bt_gather(const Geom& g, int c0, int ncol, const double* psi, long long bstride, double* R,
                             cudaStream_t st);
// Host: the rank-k basis of R (bt.cu) — W = Qᵀ R (k × pitch) and
// U_m = Q (W Q)^m (nE × kp each, m < nmat); -1 if the rank reaches kmax.
struct BtLowRank {
    int k = 0, kp = 0, sp = 0;
    std::vector<double> W, U;
    std::vector<double> Ws;   // W folded with get_bc!'s averaging of the line samples (k × sp)
};
int bt_lowrank(const std::vector<double>& R, int nx, int ny, int nmat, double tol, int kmax, BtLowRank& out);

// Base flux of a moving grid (base_flux!, timestepping.jl:273-318): on level
// spacing hc, q0x = YY·(−hc Ω) + hc Ux0 at every x-flux of row J and
// q0y = XX·(hc Ω) + hc Uy0 at every y-flux of column I, with the face
// coordinates of models.jl:145-152, YY = ((J − ½ − ny/2) hc + (ny/2) h − offy) − yc
// and XX likewise in x.  (Ω, Ux0, Uy0) of the running step are row *step of
// `tab`, `step` being the per-step counter the force kernel advances.  The
// reference evaluates these without fused multiply-adds; so does this.
struct MovingFlux {
    const double* tab = nullptr;   // [steps][3]: Ω, Ux0, Uy0; nullptr: uniform base flux
    const int* step = nullptr;
    double h = 0, offx = 0, offy = 0, xc = 0, yc = 0;
};

__device__ __forceinline__ const double* moving_row(const MovingFlux& m) { return m.tab + 3 * (*m.step); }

// q0 of x-flux row J (1-based) and of y-flux column I (1-based) on spacing hc
__device__ __forceinline__ double moving_q0x(const MovingFlux& m, const double* r, int J, int ny, double hc) {
    const double y = __dadd_rn(__dadd_rn(__dmul_rn((J - 0.5) - 0.5 * ny, hc), __dmul_rn(0.5 * ny, m.h)), -m.offy);
    return __dadd_rn(__dmul_rn(__dadd_rn(y, -m.yc), __dmul_rn(-hc, r[0])), __dmul_rn(hc, r[1]));
}
__device__ __forceinline__ double moving_q0y(const MovingFlux& m, const double* r, int I, int nx, double hc) {
    const double x = __dadd_rn(__dadd_rn(__dmul_rn((I - 0.5) - 0.5 * nx, hc), __dmul_rn(0.5 * nx, m.h)), -m.offx);
    return __dadd_rn(__dmul_rn(__dadd_rn(x, -m.xc), __dmul_rn(hc, r[0])), __dmul_rn(hc, r[2]));
}

// Stencil kernels (stencil.cu)
struct RhsArgs {
    const double* G; SlabMap Gmap;        // state Γ (all levels)
    const double* q;                      // state q, nq per level
    const double* Nprev;                  // nonlin from the previous step
    double* Nnew;                         // nonlin of this step
    double* rhs;                          // right-hand side of the trial solve
    double q0x[8], q0y[8];                // uniform base flux per level
    double fac_bc[8];                     // 0.25 dt / (Re hc²)
    double c_lap[8];                      // dt / (2 Re hc²)
    double nl_scale[8];                   // 1 / (4 hc²)
    double b1dt, b2dt;                    // β1 dt, β2 dt
    int mg;
    // linearised problem (set: GB non-null): base Γ, base q and its base flux
    const double* GB;
    const double* qB;
    double q0Bx[8], q0By[8];
    MovingFlux mv;                        // moving grid: per-face q0 replaces q0x/q0y
};
cudaError_t launch_trial_rhs(const Geom& g, const RhsArgs& a, cudaStream_t st);
// The trial right-hand sides of nsim simulations of one grid in one launch
// (batch groups): ga[s] holds simulation s's arguments (device memory), a0
// those of simulation 0 (mg and the launch shape).
cudaError_t launch_trial_rhs_group(const Geom& g, const RhsArgs& a0, const RhsArgs* ga, int nsim, cudaStream_t st);

cudaError_t launch_coarsify(const Geom& g, double* G, SlabMap fine_map, SlabMap coarse_map,
                            int nslabs, cudaStream_t st);
// FP64 residual of vort2flux! on every level of nsim simulations (mg slabs
// each, consecutive in G, psi and r), stored in FP32 into r (stencil.cu).
cudaError_t launch_resid_lap(const Geom& g, const double* G, const double* psi, float* r, int nsim, cudaStream_t st);

struct CurlArgs {
    const double* psi; SlabMap psi_map;
    const double* coarse; SlabMap coarse_map;  // coarser level ψ, or nullptr
    double* q; long long q_bstride, q_lstride; int q_lev0;
    int nlev;                                  // levels in this launch
    int nbatch;
    int mg;                                    // for "is coarsest" test
};
cudaError_t launch_curl(const Geom& g, const CurlArgs& a, cudaStream_t st);

// Body / coupling kernels (body.cu)
struct BodyDev {
    int nb, nf, nbodies;
    const double* xb;       // (nb, 2) column-major
    const double* ds;       // nb
    const int* bidx;        // (nb, 2) column-major, Julia 1-based floor((x+off)/h)
    double* w;              // [nf][13][13] weights (k-major, x components then y)
    const int* body_start;  // nbodies + 1 prefix of points
    // E' then C' as a sorted segmented reduction
    int n_src;              // Γ points in the support of C'E'
    const int* src_pts;     // [n_src] flat (j * P + i) offsets into a slab
    const int* src_rows;    // [n_src * 4] flux rows (index into et_ptr) or -1
    const int* et_ptr;      // CSR row pointer over touched flux points
    const int* et_k;        // CSR: force component index (0..nf-1), sorted ascending
    const int* et_w;        // CSR: index into w[]
    int n_et_rows;          // touched flux points
    const int* et_flux;     // [n_et_rows] level-1 flux index of each CSR row
};
cudaError_t launch_weights(const Geom& g, double h, double offx, double offy,
                           const BodyDev& b, cudaStream_t st);
cudaError_t launch_E(const Geom& g, const BodyDev& b, const double* q, long long q_stride,
                     int nbatch, double q0x, double q0y, double* F, long long F_stride,
                     cudaStream_t st, const MovingFlux& mv = MovingFlux{}, const double* ub = nullptr,
                     double hub = 0.0);
// Moving bodies (MotionFunction): kinematics from the step's motion-table row,
// the projection source in gather form, and the singular-B flag.
cudaError_t launch_kinematics(const Geom& g, const BodyDev& b, const double* x0, const double* tab, const int* step,
                              double h, double offx, double offy, double* xb, int* bidx, double* ub, int* bbox,
                              int* status, cudaStream_t st);
cudaError_t launch_proj_src_moving(const Geom& g, const BodyDev& b, const double* Fb, const int* bbox, double* Gsrc,
                                   cudaStream_t st);
cudaError_t launch_info_to_status(const int* info, int* status, cudaStream_t st);
cudaError_t launch_gemv(const double* A, const double* x, double* y, int n, cudaStream_t st);
// The force history holds hist_cap steps: a step past it writes nothing and
// sets bit 3 of *status.
cudaError_t launch_stress(const BodyDev& b, const double* Fb, double h, double dt,
                          double* hist, int hist_cap, int* counter, int* status, cudaStream_t st);
cudaError_t launch_proj_src(const Geom& g, const BodyDev& b, const double* Fb, double* Gsrc,
                            cudaStream_t st);
// launch_stress and launch_proj_src in one launch (fixed bodies)
cudaError_t launch_stress_src(const BodyDev& b, const double* Fb, double h, double dt, double* hist, int hist_cap,
                              int* counter, int* status, double* Gsrc, cudaStream_t st);
cudaError_t launch_unit_src(const Geom& g, const BodyDev& b, int col0, int ncol, double* G,
                            long long bstride, cudaStream_t st);

// Dense linear algebra (linalg.cu): in-place inverse by Gauss–Jordan with
// partial pivoting of the row-major n×n matrix A; `work` holds
// gj_work_doubles(n) doubles and `info` one int (set to the failing column + 1
// on a zero pivot).
// From n = 513 on the elimination runs panel by panel (64 columns), each
// panel as one rank-64 update of the augmented matrix.
cudaError_t launch_gj_inverse(double* A, int n, double* work, int* info, cudaStream_t st);
size_t gj_work_doubles(int n);   // doubles of `work` for launch_gj_inverse

// ---------------------------------------------------------------------------
// Discrete adjoint of the step (adjoint.cu)
// ---------------------------------------------------------------------------
cudaError_t launch_adj_curlT(const Geom& g, const double* qb, const double* prev_bc, const double* prev_W,
                             double* psib, double* bc_out, cudaStream_t st);
cudaError_t launch_adj_coarsifyT(const Geom& g, double* G, long long lstride, int lev, int zero_lev,
                                 cudaStream_t st);
cudaError_t launch_zero_centre(const Geom& g, double* G, cudaStream_t st);
cudaError_t launch_adj_E_rotT(const Geom& g, const BodyDev& b, const double* W, double wx, double wy,
                              const double* stepw, const int* adj_n, double* Ft, cudaStream_t st);
cudaError_t launch_gemv_t(const double* A, const double* x, double* y, int n, cudaStream_t st);
cudaError_t launch_adj_Et(const Geom& g, const BodyDev& b, const double* Fbar, double* qsb, double* acc,
                          cudaStream_t st);
// Trial-step adjoint: see adjoint.cu.
struct AdjTrialArgs {
    const double* rb;          // r̄ = A⁻¹ Γ̄s, mg slabs
    const double* Nb_in;       // N̄ of the next state, mg slabs
    double* Nb_out;            // N̄ of this state (β2 dt r̄)
    const double* tapeG;       // forward Γ_n, mg slabs per tape slot
    const double* tapeq;       // forward q_n, nq·mg per tape slot
    long long tape_gstride, tape_qstride;
    const int* adj_n;          // current step n (tape slot n % k)
    int k;
    double* Gb;                // out: Γ̄_n
    double* qb;                // out: q̄_n (nq per level)
    double* bcv;               // edge adjoints per level (mg·nbc)
    double* q0part;            // per-block partial sums of Σq̄0 [block][2]
    double q0x[8], q0y[8];
    double c_lap[8], fac_bc[8], nl_scale[8];
    double b1dt, b2dt;
    int mg;
};

int adj_nlq_blocks(const Geom& g);
cudaError_t launch_adj_trial(const Geom& g, const AdjTrialArgs& a, cudaStream_t st);
cudaError_t launch_adj_tick(int* adj_n, cudaStream_t st);
// Body-point position gradient (body.cu, adjoint.cu): derivative weights
// wd[nf][2][169] once, then per adjoint step
//   gxb[p] += Σ_{kk ∈ {p, nb+p}} ∇_p [ F̄_kk (E(q_{n+1,1} + q0))_kk − F̃_n,kk (E C r̄₁)_kk ]
// with F̃_n and q_{n+1,1} read from tape slot (*adj_n) % k.
cudaError_t launch_dweights(double h, double offx, double offy, const BodyDev& b, double* wd, cudaStream_t st);
struct AdjXbArgs {
    const double* wd;
    const double* Fbar;        // F̄ = B⁻ᵀ F̃̄ of this step
    const double* tapeFb;      // [k][nf]
    const double* tapeq1;      // [k][nq]: level-1 q after each step
    const int* adj_n; int k;
    double q0x, q0y;           // level-1 base flux
    const double* rb1;         // r̄ on level 1 (one slab)
    double* gxb;               // (nb, 2) column-major accumulator
};
cudaError_t launch_adj_xb(const Geom& g, const BodyDev& b, const AdjXbArgs& a, cudaStream_t st);

}  // namespace ibpm
