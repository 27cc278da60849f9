// C ABI of libibpm_gpu.so: problem setup, state transfer and the time step
// advance!(state, prob, t) of src/timestepping/timestepping.jl:35-67 for
// static bodies, run as CUDA-graph replays of hand-written sm_100a kernels.
#include "../../include/ibpm_gpu.h"
#include "ibpm_internal.cuh"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

using namespace ibpm;

#define IBPM_VERSION_STR "ibpm_gpu 0.1.0 (sm_100a, FP64)"

// FP32_REFINED: steps after create or set_state that run one more correction
// sweep per solve.  The first lacks good initial guesses (ψ and the previous
// projection may not belong to the state); the next ones follow an impulsive
// start, whose per-step changes are orders of magnitude above the later ones.
// With 8 such steps the largest one-sweep CD error of the two-cylinder 1024²
// start (dt = 0.001) fell at step 11, 1.7e-6; it decays below 1.2e-7 by step
// 100.  32 steps cover that transient for a few ms per state change.
static const int kColdSteps = 32;

struct ibpm_handle {
    int device = 0;
    cudaStream_t st = nullptr;
    Geom g;
    double h = 0, offx = 0, offy = 0, Re = 0, dt = 0, Ux = 0, Uy = 0, incl = 0;
    double beta[2] = {1.5, -0.5};
    int nb = 0, nf = 0, nbodies = 0;
    std::vector<int> body_start;
    DstPlan px{}, py{};
    bool have_px = false, have_py = false;
    // state
    double* G[2] = {nullptr, nullptr};     // Γ (ping-pong: state / trial)
    double* Nl[2] = {nullptr, nullptr};    // nonlinear term (ping-pong)
    int cur = 0;                           // parity: G[cur], Nl[cur] hold the state
    double* psi = nullptr;                 // ψ, mg slabs
    double* q = nullptr;                   // q, (nq, mg) reference layout
    double* qs = nullptr;                  // trial flux, level 1 only
    double* rhs = nullptr;                 // mg slabs of scratch
    double* Gsrc = nullptr;                // projection source, one slab, zero off-support
    double* F = nullptr;                   // E (qs + q0)
    double* Fb = nullptr;                  // F̃b
    double* Binv = nullptr;                // nf×nf row-major
    double* nonlin1_shadow = nullptr;      // nonlin[1] as set, until the next step
    bool nonlin1_valid = false;
    double q0x[8] = {0}, q0y[8] = {0};
    // body
    double* d_xb = nullptr; double* d_ds = nullptr; int* d_bidx = nullptr; double* d_w = nullptr;
    int* d_body_start = nullptr;
    int* d_src_pts = nullptr; int* d_src_rows = nullptr; int* d_et_ptr = nullptr; int* d_et_k = nullptr;
    int* d_et_w = nullptr; int* d_et_flux = nullptr;
    BodyDev body{};
    // per-step outputs
    double* hist = nullptr; int hist_cap = 0;
    double* pin_hist = nullptr;            // page-locked host mirror of hist (the advance read-back)
    int* pin_status = nullptr;             // page-locked host copy of *status
    int* counter = nullptr; int* status = nullptr;
    cudaGraphExec_t gexec[2] = {nullptr, nullptr};
    cudaGraphExec_t gcold[2] = {nullptr, nullptr};  // FP32_REFINED: first step after a state change
    bool graphs_ready = false;
    // FP32_REFINED
    int prec = IBPM_PREC_FP64;
    int sweeps = 1;                        // correction sweeps per solve
    int cold = kColdSteps;                 // steps left that lack good initial guesses
    float* T32 = nullptr;                  // mg slabs of FP32 transform scratch
    double* Pp = nullptr;                  // A⁻¹C'E'F̃b of the previous step (level 1)
    // boundary-transfer vort2flux! (bt.cu; mg >= 2): R = get_bc!∘Δ⁻¹∘apply_bc!
    // (its rank-k factors), the edge vectors, the line samples (FP64 in both
    // precisions) and the edge part of the x-spectrum of every level
    bool bt = false;                       // the step runs the boundary transfer
    int chain = IBPM_CHAIN_BOUNDARY_TRANSFER;  // the level chain set (one level: no effect)
    int bt_k = 0, bt_kp = 0;               // rank of R's basis and its pitch
    double *btW = nullptr, *btU = nullptr, *btP = nullptr, *btE = nullptr, *btS = nullptr, *btY = nullptr;
    float* btY32 = nullptr;                // the FP32 edge part (FP32_REFINED)
    // linearised problem (ibpm_set_base_state): base Γ, base q, base flux
    bool lin = false;
    double* GB = nullptr;
    double* qB = nullptr;
    double q0Bx[8] = {0}, q0By[8] = {0};
    // moving grid (ibpm_set_moving_grid): per-step (Ω, Ux0, Uy0) rows indexed by `counter`
    bool moving = false;
    double mv_xc = 0, mv_yc = 0;
    double mv_last[3] = {0, 0, 0};         // the row of the last step run (or of t = 0)
    double* mtab = nullptr; int mtab_cap = 0;
    // moving bodies (ibpm_set_motion_function): per-step rows (x, y, cos θ, sin θ, ẋ, ẏ, θ̇, ·) per body
    bool bodies_moving = false;
    double* d_x0 = nullptr;                // reference points (nb, 2)
    double* d_ub = nullptr;                // body-point velocities (nb, 2)
    int* d_bbox = nullptr;                 // min/max body_idx of the step
    double* btab = nullptr; int btab_cap = 0;
    double *bGB = nullptr, *bPB = nullptr, *bQB = nullptr, *bwork = nullptr;  // per-step B rebuild
    int* binfo = nullptr;
    // discrete adjoint (allocated by the first ibpm_adjoint_run)
    int adj_k = 0, adj_ncp = 0, adj_nsteps = 0;
    double* tapeG = nullptr;               // [k][mg slabs]  Γ_n of the segment being reversed
    double* tapeq = nullptr;               // [k][nq·mg]      q_n
    double* ck = nullptr;                  // checkpoints (and the final state), ck_doubles each
    long long ck_doubles = 0;
    std::vector<int> ck_cur, ck_cold;
    double* Gb = nullptr;                  // Γ̄ (mg slabs)
    double* qb = nullptr;                  // q̄ (nq·mg)
    double* Nb[2] = {nullptr, nullptr};    // N̄ (ping-pong)
    double* Gt = nullptr;                  // Γ̄' and Γ̄s (mg slabs)
    double* psib = nullptr;                // ψ̄ of one level
    double* Wadj = nullptr;                // solve results of the adjoint level chain (mg slabs)
    double* rb = nullptr;                  // r̄ = A⁻¹ Γ̄s (mg slabs)
    double* qsb = nullptr;                 // q̄s (nq)
    double* Ft = nullptr; double* Fbar = nullptr;
    double* bcc = nullptr; double* bcv = nullptr;  // edge adjoints (mg·nbc each)
    double* q0part = nullptr;              // [mg][blocks][2] + 2 (E' part)
    double* stepw = nullptr;               // objective weight of each step
    int* adj_n = nullptr;
    double adj_wx = 0, adj_wy = 0;
    cudaGraphExec_t gadj[2] = {nullptr, nullptr};
    // body-point position gradient (ibpm_adjoint_run with grad_xb)
    bool adj_xb = false;                   // requested by the current run
    bool gadj_xb = false;                  // the captured adjoint graphs include it
    double* wd = nullptr;                  // [nf][2][169] position derivatives of the weights
    double* tapeFb = nullptr;              // [k][nf]  F̃b of each step of the segment
    double* tapeq1 = nullptr;              // [k][nq]  level-1 q after each step
    double* gxb = nullptr;                 // (nb, 2) accumulator
    int xb_k = 0;
    // batch groups (ibpm_batch_create): members of one grid and precision keep
    // their step fields in group arenas, member after member, so that while a
    // group's step is captured its first member stands for all `gsim` of them:
    // every transform and stencil launch covers the slabs of all, and the body
    // operators (E, B⁻¹, update_stress!) run per member on branch streams
    bool in_batch = false;                 // released with its batch only
    bool arena = false;                    // step fields live in a group arena
    int gsim = 1;
    ibpm_handle* const* gmem = nullptr;    // the group's members (this one first)
    const double* g_den = nullptr;         // [gsim][9]: 2 Re hc² per level, then dt
    const double* g_cA = nullptr;          // [gsim]: dt / (2 Re h²)
    const RhsArgs* g_rhs[2] = {nullptr, nullptr};  // [gsim] trial right-hand side arguments per parity
    cudaStream_t* g_br = nullptr;          // [gsim] branch streams
    cudaEvent_t* g_ev = nullptr;           // [gsim + 1] fork and join events
    // measurement
    int launches = 0;                      // kernel launches enqueued (counted always)
    bool prof_on = false;                  // eager profiling: events around every launch
    std::vector<cudaEvent_t> prof_ev;      // start/stop pairs
    std::vector<int> prof_lab;
    std::vector<double> prof_bytes;
    int prof_n = 0;
    void* flush_buf = nullptr;             // > L2, written between timed steps
    size_t flush_bytes = 0;
    std::string err;
};

static std::string g_create_err;

// Programmatic dependent launch for the step's kernels (IBPM_NO_PDL=1 turns it off).
bool ibpm::pdl_enabled() {
    static const bool on = [] {
        const char* e = getenv("IBPM_NO_PDL");
        return !(e && e[0] == '1');
    }();
    return on;
}
static const int kBChunk = 128;  // columns of B built per batch

void ibpm::set_global_error(const char* msg) { g_create_err = msg ? msg : ""; }

#define CK(call)                                                                              \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess) {                                                              \
            h->err = std::string(#call) + ": " + cudaGetErrorString(e_);                      \
            return IBPM_ERR_CUDA;                                                             \
        }                                                                                     \
    } while (0)

// Kernel classes reported by ibpm_profile (order of IBPM_KERNEL_* in the header).
static const char* kKernelNames[] = {"trial_rhs", "dst_x", "dst_y", "coarsify", "curl",
                                     "E_gather", "binv_gemv", "stress", "proj_src", "adjoint",
                                     "resid", "bt_chain"};
enum { K_RHS = 0, K_DSTX, K_DSTY, K_COARSIFY, K_CURL, K_E, K_GEMV, K_STRESS, K_SRC, K_ADJ, K_RESID, K_BTCHAIN,
       K_COUNT };

static int prof_pre(ibpm_handle* h, int label, double bytes) {
    ++h->launches;
    if (!h->prof_on) return -1;
    const int i = h->prof_n++;
    if ((int)h->prof_ev.size() < 2 * (i + 1)) return -1;  // events are created before capture
    h->prof_lab.push_back(label);
    h->prof_bytes.push_back(bytes);
    // an event record node when captured (a plain record only orders a capture)
    cudaEventRecordWithFlags(h->prof_ev[2 * i], h->st, cudaEventRecordExternal);
    return i;
}
static void prof_post(ibpm_handle* h, int i) {
    if (i >= 0) cudaEventRecordWithFlags(h->prof_ev[2 * i + 1], h->st, cudaEventRecordExternal);
}
// Launch `call` (a cudaError_t expression) as kernel class `label` moving
// `bytes` algorithmic bytes.
#define LAUNCH(label, bytes, call)                 \
    do {                                           \
        const int pi_ = prof_pre(h, label, bytes); \
        CK(call);                                  \
        prof_post(h, pi_);                         \
    } while (0)

static int fail(ibpm_handle* h, int code, const std::string& msg) {
    h->err = msg;
    return code;
}

template <class T>
static int dalloc(ibpm_handle* h, T** p, size_t n) {
    if (n == 0) n = 1;
    cudaError_t e = cudaMalloc((void**)p, n * sizeof(T));
    if (e != cudaSuccess) {
        *p = nullptr;
        h->err = std::string("cudaMalloc: ") + cudaGetErrorString(e);
        return IBPM_ERR_NOMEM;
    }
    return IBPM_OK;
}

static SlabMap levmap(const Geom& g, int lev0, int nlev, long long bstride = 0) {
    SlabMap m;
    m.nlev = nlev; m.lev0 = lev0; m.lstride = g.S; m.bstride = bstride ? bstride : g.S * g.mg;
    return m;
}

static SpecParams spec(const ibpm_handle* h, int mode, int f32 = 0) {
    SpecParams sp;
    sp.mode = mode;
    sp.f32 = f32;
    sp.scale = 1.0 / (4.0 * h->g.nx * h->g.ny);  // laplacian.jl:38
    sp.dt = h->dt;
    for (int l = 0; l < 8; ++l) {
        const double hc = h->h * std::ldexp(1.0, l);
        sp.den[l] = 2.0 * h->Re * (hc * hc);       // laplacian.jl:69
    }
    sp.mden = h->gsim > 1 ? h->g_den : nullptr;
    return sp;
}

// One Poisson-type solve x = S((S b) ./ M .* scale) on the slabs of `map`:
// x-pass (b → tmp), y-pass with the spectral divide (tmp in place), x-pass
// (tmp → out, stored or subtracted).  b may equal tmp; tmp may equal out.
static int poisson(ibpm_handle* h, const double* b, SlabMap bmap, double* tmp, SlabMap tmap, double* out,
                   SlabMap omap, int nslabs, int mode, int emit, const double* coarse = nullptr,
                   SlabMap cmap = SlabMap{}) {
    const Geom& g = h->g;
    XPassArgs a{};
    a.in = b; a.out = tmp; a.in_map = bmap; a.out_map = tmap;
    a.coarse = coarse; a.coarse_map = cmap;
    a.nslabs = nslabs; a.line0 = 0; a.line1 = g.n2;
    a.load = coarse ? XLOAD_BC : XLOAD_PLAIN; a.emit = XEMIT_STORE;
    const double slab_bytes = 16.0 * g.n1 * g.n2 * nslabs;  // read + write every element once
    LAUNCH(K_DSTX, slab_bytes, launch_dst_x(g, h->px, a, h->st));
    LAUNCH(K_DSTY, slab_bytes, launch_dst_y(g, h->py, h->px, tmp, tmap, nslabs, spec(h, mode), h->st));
    XPassArgs c{};
    c.in = tmp; c.out = out; c.in_map = tmap; c.out_map = omap;
    c.nslabs = nslabs; c.line0 = 0; c.line1 = g.n2;
    c.load = XLOAD_PLAIN; c.emit = emit;
    LAUNCH(K_DSTX, slab_bytes * (emit == XEMIT_SUB ? 1.5 : 1.0), launch_dst_x(g, h->px, c, h->st));
    return IBPM_OK;
}

static double c_lap(const ibpm_handle* h, int lev) {
    const double hc = h->h * std::ldexp(1.0, lev);
    return h->dt / (2.0 * h->Re * (hc * hc));  // laplacian.jl:69
}

// The moving grid's base flux for the kernels, or none (uniform q0x, q0y).
static MovingFlux mv_of(const ibpm_handle* h) {
    MovingFlux m;
    if (!h->moving) return m;
    m.tab = h->mtab; m.step = h->counter;
    m.h = h->h; m.offx = h->offx; m.offy = h->offy; m.xc = h->mv_xc; m.yc = h->mv_yc;
    return m;
}

// (Ω, Ux0, Uy0) of base_flux! for a MovingGrid (timestepping.jl:283-296) from
// the motion's U, V, θ, θ̇ at the step's t and the problem's free stream.
static void moving_rates(const ibpm_handle* h, const double* m, double* r) {
    const double U = m[0], V = m[1], a = -m[2];
    double Ux0 = U * std::cos(a) - V * std::sin(a);
    double Uy0 = U * std::sin(a) + V * std::cos(a);
    Ux0 += h->Ux * std::cos(h->incl) - h->Uy * std::sin(h->incl);
    Uy0 += h->Ux * std::sin(h->incl) + h->Uy * std::cos(h->incl);
    r[0] = -m[3]; r[1] = Ux0; r[2] = Uy0;
}

// update_stress! (timestepping.jl:330-354) and the projection source C'E'F̃b
// on level 1: for fixed bodies one launch (block 0 reduces CD/CL, the others
// gather the sorted contributor lists); for moving bodies the stress kernel
// and the gather form over the moved points.
static int stress_and_src(ibpm_handle* h) {
    if (h->bodies_moving) {
        LAUNCH(K_STRESS, 8.0 * 3 * h->nb,
               launch_stress(h->body, h->Fb, h->h, h->dt, h->hist, h->hist_cap, h->counter, h->status, h->st));
        LAUNCH(K_SRC, 8.0 * 4 * 169 * h->nf, launch_proj_src_moving(h->g, h->body, h->Fb, h->d_bbox, h->Gsrc, h->st));
        return IBPM_OK;
    }
    LAUNCH(K_SRC, 8.0 * (4 * 169 * h->nf + 3 * h->nb),
           launch_stress_src(h->body, h->Fb, h->h, h->dt, h->hist, h->hist_cap, h->counter, h->status, h->Gsrc, h->st));
    return IBPM_OK;
}

// Run `fn` for every member of the group being captured (the handle alone
// outside groups), each member on its own branch stream forked from and
// joined back into the lead's stream.
template <class F>
static int per_member(ibpm_handle* h, F fn) {
    if (h->gsim <= 1) return fn(h);
    CK(cudaEventRecord(h->g_ev[0], h->st));
    for (int i = 0; i < h->gsim; ++i) {
        ibpm_handle* m = h->gmem[i];
        cudaStream_t own = m->st;
        CK(cudaStreamWaitEvent(h->g_br[i], h->g_ev[0], 0));
        m->st = h->g_br[i];
        const int rc = fn(m);
        m->st = own;
        if (rc) {
            if (m != h) h->err = m->err;
            return rc;
        }
        CK(cudaEventRecord(h->g_ev[1 + i], h->g_br[i]));
        CK(cudaStreamWaitEvent(h->st, h->g_ev[1 + i], 0));
    }
    return IBPM_OK;
}

// boundary_forces! (timestepping.jl:154-163) of one simulation: F = E(qs + q0),
// F̃b = B⁻¹ F, then update_stress! and the projection source.
static int forces_and_src(ibpm_handle* h) {
    const Geom& g = h->g;
    LAUNCH(K_E, 16.0 * 169 * h->nf, launch_E(g, h->body, h->qs, 0, 1, h->q0x[0], h->q0y[0], h->F, h->nf, h->st, mv_of(h),
                    h->bodies_moving ? h->d_ub : nullptr, h->h));
    LAUNCH(K_GEMV, 8.0 * h->nf * (h->nf + 2.0), launch_gemv(h->Binv, h->F, h->Fb, h->nf, h->st));
    return stress_and_src(h);
}

static RhsArgs rhs_args(const ibpm_handle* h, int p) {
    const Geom& g = h->g;
    RhsArgs ra{};
    ra.G = h->G[p]; ra.Gmap = levmap(g, 0, g.mg); ra.q = h->q;
    ra.Nprev = h->Nl[p]; ra.Nnew = h->Nl[p ^ 1];
    for (int l = 0; l < g.mg; ++l) {
        const double hc = h->h * std::ldexp(1.0, l);
        ra.q0x[l] = h->q0x[l]; ra.q0y[l] = h->q0y[l];
        ra.fac_bc[l] = 0.25 * h->dt / (h->Re * (hc * hc));
        ra.c_lap[l] = c_lap(h, l);
        ra.nl_scale[l] = 1.0 / (4.0 * (hc * hc));
    }
    ra.b1dt = h->beta[0] * h->dt; ra.b2dt = h->beta[1] * h->dt; ra.mg = g.mg;
    ra.mv = mv_of(h);
    if (h->lin) {
        ra.GB = h->GB; ra.qB = h->qB;
        for (int l = 0; l < g.mg; ++l) { ra.q0Bx[l] = h->q0Bx[l]; ra.q0By[l] = h->q0By[l]; }
    }
    return ra;
}

// vort2flux! (curl.jl:133-165) on `nbatch` independent fields G (slab-major,
// batch stride bstride), level by level as the reference: coarsify chain,
// Δ⁻¹ solves from the coarsest level inwards with the edge values of the next
// coarser ψ, then q = curl ψ on levels [qlev0, qlev0 + qnlev) into q (nq per
// level, batch stride q_bstride).
static int vort2flux(ibpm_handle* h, double* G, double* psi, long long bstride, int nbatch, double* q,
                     long long q_bstride, int qlev0, int qnlev) {
    const Geom& g = h->g;
    const int mg = g.mg;
    for (int lev = 1; lev < mg; ++lev)
        LAUNCH(K_COARSIFY, 8.0 * 1.25 * g.n1 * g.n2 * nbatch,
               launch_coarsify(g, G, levmap(g, lev - 1, 1, bstride), levmap(g, lev, 1, bstride), nbatch, h->st));
    for (int lev = mg - 1; lev >= 0; --lev) {
        SlabMap m = levmap(g, lev, 1, bstride);
        const double* coarse = (lev < mg - 1) ? psi : nullptr;
        int rc = poisson(h, G, m, psi, m, psi, m, nbatch, SPEC_DELTA, XEMIT_STORE, coarse,
                         levmap(g, lev + 1, 1, bstride));
        if (rc) return rc;
    }
    CurlArgs ca{};
    ca.psi = psi; ca.psi_map = levmap(g, qlev0, qnlev, bstride);
    ca.coarse = psi; ca.coarse_map = levmap(g, qlev0 + 1, qnlev, bstride);
    ca.q = q; ca.q_bstride = q_bstride; ca.q_lstride = g.nq; ca.q_lev0 = qlev0;
    ca.nlev = qnlev; ca.nbatch = nbatch; ca.mg = mg;
    LAUNCH(K_CURL, 8.0 * ((double)g.n1 * g.n2 + g.nq) * qnlev * nbatch, launch_curl(g, ca, h->st));
    return IBPM_OK;
}

// ---------------------------------------------------------------------------
// Boundary-transfer vort2flux! (ibpm_internal.cuh, bt.cu).  The reference
// solves the levels one after another, each with the edge values of the next
// coarser ψ (curl.jl:147-162).  Here every level's interior part Δ⁻¹Γ_ℓ is
// one multi-level solve; the edge vectors follow from its line samples by the
// chain e_ℓ = get_bc!(Δ⁻¹Γ_{ℓ+1}) + R e_{ℓ+1} (mg−1 small launches); one
// y-pass builds every level's edge part from e_ℓ, and one x-pass transforms
// the sum of both parts.  The result is the reference's ψ and q up to
// rounding (both parts are the same linear operators applied in another
// order).
// ---------------------------------------------------------------------------

// R at create: the get_bc! samples of Δ⁻¹ of a unit source at every edge entry
// (FP64 solves, `chunk` columns per batch), then its rank-k basis on the host
// (bt_lowrank), used in FP64 by both precisions.  A rank that does
// not settle (never seen) leaves the handle on the level-by-level chain.
static int upload_bt(ibpm_handle* h, const BtLowRank& lr);

// R depends only on (nx, ny) and each mg needs its own U_m: handles of one
// size (finite-difference runs, batch members) share the host factors.
struct BtCacheKey {
    int nx, ny, mg;
    bool operator<(const BtCacheKey& o) const {
        return nx != o.nx ? nx < o.nx : ny != o.ny ? ny < o.ny : mg < o.mg;
    }
};
static std::mutex g_bt_mutex;
static std::map<BtCacheKey, std::shared_ptr<const BtLowRank>> g_bt_cache;

static int build_bt(ibpm_handle* h) {
    const Geom& g = h->g;
    if (g.mg < 2) return IBPM_OK;
    const int nE = bt_edge_len(g), ep = bt_edge_pitch(g);
    const int mg = g.mg;
    int rc;
    std::shared_ptr<const BtLowRank> cached;
    {
        std::lock_guard<std::mutex> lock(g_bt_mutex);
        auto it = g_bt_cache.find(BtCacheKey{g.nx, g.ny, mg});
        if (it != g_bt_cache.end()) cached = it->second;
    }
    if (cached) return upload_bt(h, *cached);
    double *R = nullptr, *GB = nullptr;
    const int chunk = std::min(nE, kBChunk);
    if ((rc = dalloc(h, &R, (size_t)nE * ep)) || (rc = dalloc(h, &GB, (size_t)g.S * chunk))) {
        cudaFree(R);
        return rc;
    }
    SlabMap one = levmap(g, 0, 1, g.S);
    cudaError_t e = cudaMemsetAsync(R, 0, sizeof(double) * nE * ep, h->st);
    for (int c0 = 0; c0 < nE && rc == IBPM_OK && e == cudaSuccess; c0 += chunk) {
        const int ncol = std::min(chunk, nE - c0);
        e = cudaMemsetAsync(GB, 0, sizeof(double) * g.S * ncol, h->st);
        if (e == cudaSuccess) e = launch_bt_unit_src(g, c0, ncol, GB, g.S, h->st);
        if (e == cudaSuccess) rc = poisson(h, GB, one, GB, one, GB, one, ncol, SPEC_DELTA, XEMIT_STORE);
        if (e == cudaSuccess && rc == IBPM_OK) e = launch_bt_gather(g, c0, ncol, GB, g.S, R, h->st);
    }
    std::vector<double> Rh((size_t)nE * ep);
    if (e == cudaSuccess && rc == IBPM_OK)
        e = cudaMemcpyAsync(Rh.data(), R, sizeof(double) * Rh.size(), cudaMemcpyDeviceToHost, h->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->st);
    cudaFree(GB);
    cudaFree(R);
    if (rc) return rc;
    if (e != cudaSuccess) return fail(h, IBPM_ERR_CUDA, std::string("R setup: ") + cudaGetErrorString(e));
    auto lr = std::make_shared<BtLowRank>();
    if (bt_lowrank(Rh, g.nx, g.ny, std::max(0, mg - 2), 1e-14, std::min(nE, 1024), *lr)) return IBPM_OK;
    {
        std::lock_guard<std::mutex> lock(g_bt_mutex);
        g_bt_cache[BtCacheKey{g.nx, g.ny, mg}] = lr;
    }
    return upload_bt(h, *lr);
}

static int upload_bt(ibpm_handle* h, const BtLowRank& lr) {
    const Geom& g = h->g;
    const int mg = g.mg, ep = bt_edge_pitch(g);
    const bool f32 = h->prec == IBPM_PREC_FP32_REFINED;
    int rc;
    h->bt_k = lr.k;
    h->bt_kp = lr.kp;
    const size_t nw = lr.Ws.size(), nu = std::max<size_t>(1, lr.U.size()), np = (size_t)(mg - 1) * lr.kp;
    const size_t slabs = (size_t)g.S * mg, ns = (size_t)bt_sample_len(g) * mg, ne = (size_t)ep * mg;
    if ((rc = dalloc(h, &h->btW, nw)) || (rc = dalloc(h, &h->btU, nu)) || (rc = dalloc(h, &h->btP, np)) ||
        (rc = dalloc(h, &h->btE, ne)) || (rc = dalloc(h, &h->btS, ns)) || (rc = dalloc(h, &h->btY, slabs)))
        return rc;
    CK(cudaMemcpyAsync(h->btW, lr.Ws.data(), sizeof(double) * nw, cudaMemcpyHostToDevice, h->st));
    if (!lr.U.empty())
        CK(cudaMemcpyAsync(h->btU, lr.U.data(), sizeof(double) * lr.U.size(), cudaMemcpyHostToDevice, h->st));
    CK(cudaMemsetAsync(h->btP, 0, sizeof(double) * np, h->st));
    CK(cudaMemsetAsync(h->btE, 0, sizeof(double) * ne, h->st));
    CK(cudaMemsetAsync(h->btS, 0, sizeof(double) * ns, h->st));
    CK(cudaMemsetAsync(h->btY, 0, sizeof(double) * slabs, h->st));  // the coarsest slab stays zero
    if (f32) {
        if ((rc = dalloc(h, &h->btY32, slabs))) return rc;
        CK(cudaMemsetAsync(h->btY32, 0, sizeof(float) * slabs, h->st));
    }
    h->bt = true;
    return IBPM_OK;
}

// From the y-pass output Y of every level (x-spectral; FP64 or FP32): the line
// samples of levels 1 … mg−1, the edge chain down to level 0, and the edge
// part of levels 0 … nyb−1 by one y-pass, into btY / btY32.
static int bt_edges(ibpm_handle* h, const void* Y, bool f32, int nyb) {
    const Geom& g = h->g;
    const int mg = g.mg, ns = h->gsim;
    const long long bs = g.S * mg;
    const int nE = bt_edge_len(g);
    const double es = f32 ? 4.0 : 8.0;
    // the samples, the chain and the edge vectors are FP64 in both precisions
    LAUNCH(K_BTCHAIN, (es * (g.ny / 2 + 3.0) * g.n1 + 16.0 * g.n1) * (mg - 1) * ns,
           launch_dst_lines(g, h->px, Y, levmap(g, 1, mg - 1, bs), (mg - 1) * ns, h->btS, f32 ? 1 : 0, h->st));
    BtChainArgs a{};
    a.W = h->btW; a.U = h->btU; a.samples = h->btS; a.e = h->btE; a.p = h->btP;
    a.k = h->bt_k; a.kp = h->bt_kp; a.nsim = ns;
    if (mg > 2)
        LAUNCH(K_BTCHAIN, 8.0 * ((double)h->bt_k * (g.nx + g.ny + 4.0) * (1.0 + (mg - 1.0) * ns) + (mg - 1.0) * h->bt_kp * ns),
               launch_bt_project(g, a, h->st));
    LAUNCH(K_BTCHAIN, 8.0 * ((mg - 2.0) * nE * h->bt_kp + 3.0 * nE * (mg - 1) * ns), launch_bt_expand(g, a, h->st));
    BtSynth bsy{};
    bsy.e = h->btE; bsy.sx = h->px.s; bsy.nx = g.nx;
    LAUNCH(K_DSTY, es * g.n1 * g.n2 * nyb * ns,
           launch_dst_ybc(g, h->py, h->px, f32 ? (void*)h->btY32 : (void*)h->btY, levmap(g, 0, nyb, bs), nyb * ns,
                          spec(h, SPEC_DELTA, f32 ? 1 : 0), bsy, h->st));
    return IBPM_OK;
}

static int curl_levels(ibpm_handle* h, double* q, int qnlev) {
    const Geom& g = h->g;
    CurlArgs ca{};
    ca.psi = h->psi; ca.psi_map = levmap(g, 0, qnlev);
    ca.coarse = h->psi; ca.coarse_map = levmap(g, 1, qnlev);
    ca.q = q; ca.q_bstride = (long long)g.nq * g.mg; ca.q_lstride = g.nq; ca.q_lev0 = 0;
    ca.nlev = qnlev; ca.nbatch = h->gsim; ca.mg = g.mg;
    LAUNCH(K_CURL, 8.0 * ((double)g.n1 * g.n2 + g.nq) * qnlev * h->gsim, launch_curl(g, ca, h->st));
    return IBPM_OK;
}

// vort2flux! (FP64) of the handle's field G into h->psi (levels < nfull; the
// coarser ones are left as they were) and q (levels < qnlev < nfull).  The
// trial vort2flux! of a step needs only the level-1 flux, hence ψ of levels 1
// and 2; the final one recomputes every level.
static int vort2flux_bt(ibpm_handle* h, double* G, double* q, int qnlev, int nfull) {
    const Geom& g = h->g;
    const int mg = g.mg, ns = h->gsim;
    const long long bs = g.S * mg;
    const double slab = (double)g.n1 * g.n2;
    for (int lev = 1; lev < mg; ++lev)
        LAUNCH(K_COARSIFY, 8.0 * 1.25 * slab * ns,
               launch_coarsify(g, G, levmap(g, lev - 1, 1, bs), levmap(g, lev, 1, bs), ns, h->st));
    SlabMap all = levmap(g, 0, mg, bs);
    XPassArgs a{};
    a.in = G; a.out = h->rhs; a.in_map = all; a.out_map = all;
    a.nslabs = mg * ns; a.line0 = 0; a.line1 = g.n2; a.load = XLOAD_PLAIN; a.emit = XEMIT_STORE;
    LAUNCH(K_DSTX, 16.0 * slab * mg * ns, launch_dst_x(g, h->px, a, h->st));
    LAUNCH(K_DSTY, 16.0 * slab * mg * ns,
           launch_dst_y(g, h->py, h->px, h->rhs, all, mg * ns, spec(h, SPEC_DELTA), h->st));
    int rc = bt_edges(h, h->rhs, false, std::min(nfull, mg - 1));
    if (rc) return rc;
    SlabMap part = levmap(g, 0, nfull, bs);
    XPassArgs c{};
    c.in = h->rhs; c.in2 = h->btY; c.in_map = part; c.in2_map = part; c.out = h->psi; c.out_map = part;
    c.nslabs = nfull * ns; c.line0 = 0; c.line1 = g.n2; c.load = XLOAD_SUM; c.emit = XEMIT_STORE;
    LAUNCH(K_DSTX, 24.0 * slab * nfull * ns, launch_dst_x(g, h->px, c, h->st));
    return curl_levels(h, q, qnlev);
}

// vort2flux! of FP32_REFINED: `nsw` sweeps ψ ← ψ + d, the corrections d of
// every level from FP64 residuals against the present ψ (all levels read the
// ψ of before the sweep), r_ℓ = Γ_ℓ + apply_bc!(get_bc!(ψ_{ℓ+1})) − L ψ_ℓ.
// The corrections satisfy the level chain of vort2flux! themselves,
// L d_ℓ = r_ℓ + apply_bc!(get_bc!(d_{ℓ+1})), so the boundary transfer solves
// them in FP32 as above.
static int vort2flux_refined_bt(ibpm_handle* h, double* G, int nsw, double* q, int qnlev, int nfull) {
    const Geom& g = h->g;
    const int mg = g.mg;
    const long long bs = g.S * mg;
    const double slab = (double)g.n1 * g.n2;
    const int ns = h->gsim;
    for (int lev = 1; lev < mg; ++lev)
        LAUNCH(K_COARSIFY, 8.0 * 1.25 * slab * ns,
               launch_coarsify(g, G, levmap(g, lev - 1, 1, bs), levmap(g, lev, 1, bs), ns, h->st));
    SlabMap all = levmap(g, 0, mg, bs), part = levmap(g, 0, nfull, bs);
    for (int s = 0; s < nsw; ++s) {
        // the residual of every level in one stencil launch (FP32 out), then
        // its x-transform in place: a light x-pass that more CTAs share an SM with
        LAUNCH(K_RESID, (8.0 + 8.0 + 4.0) * slab * mg * ns, launch_resid_lap(g, G, h->psi, h->T32, ns, h->st));
        XPassArgs a{};
        a.in = h->T32; a.out = h->T32; a.in_map = all; a.out_map = all;
        a.nslabs = mg * ns; a.line0 = 0; a.line1 = g.n2; a.load = XLOAD_F32; a.emit = XEMIT_F32;
        LAUNCH(K_DSTX, 8.0 * slab * mg * ns, launch_dst_x(g, h->px, a, h->st));
        LAUNCH(K_DSTY, 8.0 * slab * mg * ns,
               launch_dst_y(g, h->py, h->px, h->T32, all, mg * ns, spec(h, SPEC_DELTA, 1), h->st));
        int rc = bt_edges(h, h->T32, true, std::min(nfull, mg - 1));
        if (rc) return rc;
        XPassArgs c{};
        c.in = h->T32; c.in2 = h->btY32; c.in_map = part; c.in2_map = part; c.out = h->psi; c.out_map = part;
        c.nslabs = nfull * ns; c.line0 = 0; c.line1 = g.n2; c.load = XLOAD_F32_SUM; c.emit = XEMIT_ADD;
        LAUNCH(K_DSTX, (4.0 + 4.0 + 16.0) * slab * nfull * ns, launch_dst_x(g, h->px, c, h->st));
    }
    return curl_levels(h, q, qnlev);
}

// get_trial_state!'s right-hand side of every level (of every member of the
// group being captured).
static int trial_rhs(ibpm_handle* h, int p) {
    const Geom& g = h->g;
    RhsArgs ra = rhs_args(h, p);
    ra.rhs = h->rhs;
    const double bytes = 8.0 * (4.0 * g.n1 * g.n2 + g.nq) * g.mg * h->gsim;
    if (h->gsim > 1) LAUNCH(K_RHS, bytes, launch_trial_rhs_group(g, ra, h->g_rhs[p], h->gsim, h->st));
    else LAUNCH(K_RHS, bytes, launch_trial_rhs(g, ra, h->st));
    return IBPM_OK;
}

// One step, reading the state from parity p and leaving it in parity p^1.
static int enqueue_step_fp64(ibpm_handle* h, int p) {
    const Geom& g = h->g;
    const int mg = g.mg;
    double* Gnew = h->G[p ^ 1];
    const int ns = h->gsim;
    const long long qb = (long long)g.nq * mg;
    // --- get_trial_state! (timestepping.jl:86-129)
    int rc = trial_rhs(h, p);
    if (rc) return rc;
    SlabMap all = levmap(g, 0, mg);
    rc = poisson(h, h->rhs, all, h->rhs, all, Gnew, all, mg * ns, SPEC_AINV, XEMIT_STORE);
    if (rc) return rc;
    rc = h->bt ? vort2flux_bt(h, Gnew, h->qs, 1, std::min(2, mg))  // only the level-1 trial flux is read
               : vort2flux(h, Gnew, h->psi, g.S * mg, ns, h->qs, qb, 0, 1);
    if (rc) return rc;
    // --- boundary_forces! (timestepping.jl:154-163), update_stress! (:330-354)
    if ((rc = per_member(h, forces_and_src))) return rc;
    // --- project_circ! (timestepping.jl:204-223): Γ = Γs − A⁻¹ C'E' F̃b on level 1
    SlabMap one = levmap(g, 0, 1);
    rc = poisson(h, h->Gsrc, one, h->rhs, one, Gnew, one, ns, SPEC_AINV, XEMIT_SUB);
    if (rc) return rc;
    // --- vort2flux!(state.ψ, state.q, state.Γ) (timestepping.jl:64)
    return h->bt ? vort2flux_bt(h, Gnew, h->q, mg, mg) : vort2flux(h, Gnew, h->psi, g.S * mg, ns, h->q, qb, 0, mg);
}

// ---------------------------------------------------------------------------
// FP32-refined step.  The projection solve and the final vort2flux! are
// refined: each Poisson-type solve x = M⁻¹ b (M = L for Δ⁻¹, I + cL for A⁻¹,
// L x = 4x − Σ neighbours) is one or more sweeps of
//     x ← x + S32(b − M x)
// with the residual formed in FP64 (in the first x-pass, or by one stencil
// launch over all levels) and the correction S32 = the DST-I solve in FP32,
// starting from the previous solution of the same system (ψ of the trial
// vort2flux!, the previous projection).  The error left is the FP32 error of
// the correction alone, i.e. relative to the change of x since its previous
// solution.  The trial solve and the trial vort2flux! run in FP64 (see the
// step).  The trial solve Γs = A⁻¹ rhs stays FP64: near the wall its change per step
// is O(Γ), and the force F = E(qs + q0) is a difference that cancels to
// O(dt)·|q0| there, so an FP32 error in Γs − Γ reaches CD amplified by
// |q0|/|F| (≈ 500 at dt = 0.002).  A second FP32 sweep would fix it at three
// more launches, which cost more than the FP64 solve of all levels at once.
// ---------------------------------------------------------------------------
static int correction32(ibpm_handle* h, int load, const double* b, const double* coarse, double* xg, double cA,
                        int lev, int emit, double* out) {
    const Geom& g = h->g;
    const long long bs = g.S * g.mg;
    const int ns = h->gsim;
    SlabMap m = levmap(g, lev, 1, bs);
    const double slab = (double)g.n1 * g.n2 * ns;
    XPassArgs a{};
    a.in = b; a.out = h->T32; a.in_map = m; a.out_map = m;
    a.coarse = coarse; a.coarse_map = levmap(g, lev + 1, 1, bs);
    a.aux = xg; a.aux_map = m; a.cA = cA; a.mcA = ns > 1 ? h->g_cA : nullptr;
    a.nslabs = ns; a.line0 = 0; a.line1 = g.n2; a.load = load; a.emit = XEMIT_F32;
    LAUNCH(K_DSTX, slab * (8.0 + 8.0 + 4.0), launch_dst_x(g, h->px, a, h->st));
    LAUNCH(K_DSTY, slab * 8.0,
           launch_dst_y(g, h->py, h->px, h->T32, m, ns, spec(h, load == XLOAD_RES_A ? SPEC_AINV : SPEC_DELTA, 1),
                        h->st));
    XPassArgs c{};
    c.in = h->T32; c.out = out; c.in_map = m; c.out_map = m;
    c.aux = xg; c.aux_map = m;
    c.nslabs = ns; c.line0 = 0; c.line1 = g.n2; c.load = XLOAD_F32; c.emit = emit;
    LAUNCH(K_DSTX, slab * (4.0 + 16.0 + (emit == XEMIT_ACC_SUB ? 16.0 : 0.0)), launch_dst_x(g, h->px, c, h->st));
    return IBPM_OK;
}

// vort2flux! with every level's Δ⁻¹ solve refined from the ψ in h->psi.
static int vort2flux_refined(ibpm_handle* h, double* G, int nsw, double* q, int qnlev) {
    const Geom& g = h->g;
    const int mg = g.mg;
    const long long bs = g.S * mg;
    const int ns = h->gsim;
    for (int lev = 1; lev < mg; ++lev)
        LAUNCH(K_COARSIFY, 8.0 * 1.25 * g.n1 * g.n2 * ns,
               launch_coarsify(g, G, levmap(g, lev - 1, 1, bs), levmap(g, lev, 1, bs), ns, h->st));
    int rc;
    for (int lev = mg - 1; lev >= 0; --lev) {
        const double* coarse = (lev < mg - 1) ? h->psi : nullptr;
        for (int s = 0; s < nsw; ++s) {
            if ((rc = correction32(h, XLOAD_RES_LAP, G, coarse, h->psi, 0.0, lev, XEMIT_ADD, h->psi))) return rc;
        }
    }
    CurlArgs ca{};
    ca.psi = h->psi; ca.psi_map = levmap(g, 0, qnlev, bs);
    ca.coarse = h->psi; ca.coarse_map = levmap(g, 1, qnlev, bs);
    ca.q = q; ca.q_bstride = (long long)g.nq * mg; ca.q_lstride = g.nq; ca.q_lev0 = 0;
    ca.nlev = qnlev; ca.nbatch = ns; ca.mg = mg;
    LAUNCH(K_CURL, 8.0 * ((double)g.n1 * g.n2 + g.nq) * qnlev * ns, launch_curl(g, ca, h->st));
    return IBPM_OK;
}

static int enqueue_step_refined(ibpm_handle* h, int p, int nsw) {
    const Geom& g = h->g;
    const int mg = g.mg;
    double* Gnew = h->G[p ^ 1];
    const long long bs = g.S * mg;
    const int ns = h->gsim;
    // --- get_trial_state! (FP64 trial solve: see the note above)
    int rc = trial_rhs(h, p);
    if (rc) return rc;
    SlabMap all = levmap(g, 0, mg, bs);
    rc = poisson(h, h->rhs, all, h->rhs, all, Gnew, all, mg * ns, SPEC_AINV, XEMIT_STORE);
    if (rc) return rc;
    // The trial vort2flux! in FP64, as the FP64 step runs it (the boundary
    // transfer completes only the two levels E reads).  It feeds the forces
    // directly; in FP32 with one sweep its correction error (a whole step's
    // change of ψ times the sweep's contraction, ~1e-5) moved the shedding
    // cycle's CL amplitude by 3e-6, against 2.5e-7 this way, and it cost more.
    // The final vort2flux! refines from it: levels it did not complete keep
    // the previous step's ψ and take a whole step's correction there.
    rc = h->bt ? vort2flux_bt(h, Gnew, h->qs, 1, std::min(2, mg))
               : vort2flux(h, Gnew, h->psi, g.S * mg, ns, h->qs, (long long)g.nq * mg, 0, 1);
    if (rc) return rc;
    // --- boundary_forces! and update_stress! (FP64)
    if ((rc = per_member(h, forces_and_src))) return rc;
    // --- project_circ!: P = A⁻¹ C'E' F̃b refined from the previous P; Γ[1] −= P
    for (int s = 0; s < nsw; ++s) {
        const bool last = s + 1 == nsw;
        rc = correction32(h, XLOAD_RES_A, h->Gsrc, nullptr, h->Pp, c_lap(h, 0), 0,
                          last ? XEMIT_ACC_SUB : XEMIT_ADD, last ? Gnew : h->Pp);
        if (rc) return rc;
    }
    // --- vort2flux!(state.ψ, state.q, state.Γ)
    return h->bt ? vort2flux_refined_bt(h, Gnew, nsw, h->q, mg, mg) : vort2flux_refined(h, Gnew, nsw, h->q, mg);
}

// update_bodies! for MotionFunction bodies (timestepping.jl:386-398): move the
// points to this step's row of the motion table, recompute body_idx and the
// weights of E, and rebuild B⁻¹ from B_times! (laplacian.jl:143-169) by the
// batched unit-source solves of the setup and the device Gauss–Jordan
// inverse.  The reference solves with B by conjugate gradients to reltol
// 1e-12 instead (laplacian.jl:123-141); here B⁻¹ is exact to round-off.
static int enqueue_body_update(ibpm_handle* h) {
    const Geom& g = h->g;
    const int nf = h->nf;
    LAUNCH(K_E, 8.0 * 12 * h->nb,
           launch_kinematics(g, h->body, h->d_x0, h->btab, h->counter, h->h, h->offx, h->offy, h->d_xb, h->d_bidx,
                             h->d_ub, h->d_bbox, h->status, h->st));
    LAUNCH(K_E, 8.0 * 169 * h->nf, launch_weights(g, h->h, h->offx, h->offy, h->body, h->st));
    const int chunk = std::min(nf, kBChunk);
    const long long bstride = g.S * g.mg;
    for (int c0 = 0; c0 < nf; c0 += chunk) {
        const int R = std::min(chunk, nf - c0);
        CK(cudaMemsetAsync(h->bGB, 0, sizeof(double) * bstride * R, h->st));
        LAUNCH(K_SRC, 8.0 * 196 * R, launch_unit_src(g, h->body, c0, R, h->bGB, bstride, h->st));
        SlabMap l0 = levmap(g, 0, 1, bstride);
        int rc = poisson(h, h->bGB, l0, h->bGB, l0, h->bGB, l0, R, SPEC_AINV, XEMIT_STORE);
        if (rc) return rc;
        rc = vort2flux(h, h->bGB, h->bPB, bstride, R, h->bQB, g.nq, 0, 1);
        if (rc) return rc;
        LAUNCH(K_E, 16.0 * 169 * R, launch_E(g, h->body, h->bQB, g.nq, R, 0.0, 0.0, h->Binv + c0, -(long long)nf, h->st));
    }
    LAUNCH(K_GEMV, 8.0 * 4.0 * nf * nf, launch_gj_inverse(h->Binv, nf, h->bwork, h->binfo, h->st));
    LAUNCH(K_GEMV, 8.0, launch_info_to_status(h->binfo, h->status, h->st));
    return IBPM_OK;
}

static int enqueue_step(ibpm_handle* h, int p, bool cold = false) {
    if (h->bodies_moving) {
        int rc = enqueue_body_update(h);
        if (rc) return rc;
    }
    if (h->prec == IBPM_PREC_FP32_REFINED) return enqueue_step_refined(h, p, cold ? h->sweeps + 1 : h->sweeps);
    return enqueue_step_fp64(h, p);
}

// ---------------------------------------------------------------------------
// Setup helpers
// ---------------------------------------------------------------------------
static int build_coupling(ibpm_handle* h, const ibpm_problem_desc* d) {
    const Geom& g = h->g;
    const int nb = h->nb;
    std::vector<int> bidx(2 * nb);
    for (int k = 0; k < nb; ++k) {
        // body_idx = floor((xb + off)/h) (interface-coupling.jl:86-87)
        bidx[k] = (int)std::floor((d->xb[k] + d->offx) / d->h);
        bidx[nb + k] = (int)std::floor((d->xb[nb + k] + d->offy) / d->h);
        const int bx = bidx[k], by = bidx[nb + k];
        if (bx - 6 < 1 || bx + 6 > g.nx || by - 6 < 1 || by + 6 > g.ny)
            return fail(h, IBPM_ERR_INVALID, "body point " + std::to_string(k) +
                                                 ": the 13x13 regularisation stencil leaves the finest grid");
    }
    // E' as CSR over touched flux points, contributors in ascending component order.
    std::map<int, std::vector<std::pair<int, int>>> rows;  // flux index -> (kk, widx)
    for (int kk = 0; kk < h->nf; ++kk) {
        const int comp = kk / nb, k = kk % nb;
        const int bx = bidx[k], by = bidx[nb + k];
        for (int l = 0; l < 13; ++l)
            for (int m = 0; m < 13; ++m) {
                const int I = bx + l - 6, J = by + m - 6;
                const int f = comp == 0 ? (I - 1) + (J - 1) * (g.nx + 1) : g.nu + (I - 1) + (J - 1) * g.nx;
                rows[f].push_back({kk, (kk * 13 + l) * 13 + m});
            }
    }
    std::vector<int> et_ptr, et_k, et_w, et_flux;
    std::map<int, int> row_of;
    et_ptr.push_back(0);
    for (auto& kv : rows) {
        row_of[kv.first] = (int)et_ptr.size() - 1;
        et_flux.push_back(kv.first);
        for (auto& e : kv.second) { et_k.push_back(e.first); et_w.push_back(e.second); }
        et_ptr.push_back((int)et_k.size());
    }
    // Γ points whose rot! stencil touches a regularised flux: Γ(i0, j0) uses
    // qx[i0+2, j0+1], qx[i0+2, j0+2], qy[i0+2, j0+2], qy[i0+1, j0+2] (1-based).
    auto fx = [&](int I, int J) { return (I - 1) + (J - 1) * (g.nx + 1); };
    auto fy = [&](int I, int J) { return g.nu + (I - 1) + (J - 1) * g.nx; };
    std::vector<int> src_pts, src_rows;
    for (int j0 = 0; j0 < g.n2; ++j0)
        for (int i0 = 0; i0 < g.n1; ++i0) {
            const int f4[4] = {fx(i0 + 2, j0 + 1), fx(i0 + 2, j0 + 2), fy(i0 + 2, j0 + 2), fy(i0 + 1, j0 + 2)};
            int r4[4];
            bool any = false;
            for (int r = 0; r < 4; ++r) {
                auto it = row_of.find(f4[r]);
                r4[r] = it == row_of.end() ? -1 : it->second;
                any |= r4[r] >= 0;
            }
            if (!any) continue;
            src_pts.push_back(j0 * g.P + i0);
            for (int r = 0; r < 4; ++r) src_rows.push_back(r4[r]);
        }
    int rc;
    if ((rc = dalloc(h, &h->d_xb, 2 * nb)) || (rc = dalloc(h, &h->d_ds, nb)) || (rc = dalloc(h, &h->d_bidx, 2 * nb)) ||
        (rc = dalloc(h, &h->d_w, (size_t)h->nf * 169)) || (rc = dalloc(h, &h->d_body_start, h->nbodies + 1)) ||
        (rc = dalloc(h, &h->d_src_pts, src_pts.size())) || (rc = dalloc(h, &h->d_src_rows, src_rows.size())) ||
        (rc = dalloc(h, &h->d_et_ptr, et_ptr.size())) || (rc = dalloc(h, &h->d_et_k, et_k.size())) ||
        (rc = dalloc(h, &h->d_et_w, et_w.size())) || (rc = dalloc(h, &h->d_et_flux, et_flux.size())))
        return rc;
    auto up = [&](void* dst, const void* src, size_t bytes) {
        return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, h->st);
    };
    CK(up(h->d_xb, d->xb, sizeof(double) * 2 * nb));
    CK(up(h->d_ds, d->ds, sizeof(double) * nb));
    CK(up(h->d_bidx, bidx.data(), sizeof(int) * 2 * nb));
    CK(up(h->d_body_start, h->body_start.data(), sizeof(int) * (h->nbodies + 1)));
    if (!src_pts.empty()) {
        CK(up(h->d_src_pts, src_pts.data(), sizeof(int) * src_pts.size()));
        CK(up(h->d_src_rows, src_rows.data(), sizeof(int) * src_rows.size()));
    }
    CK(up(h->d_et_ptr, et_ptr.data(), sizeof(int) * et_ptr.size()));
    CK(up(h->d_et_k, et_k.data(), sizeof(int) * et_k.size()));
    CK(up(h->d_et_w, et_w.data(), sizeof(int) * et_w.size()));
    CK(up(h->d_et_flux, et_flux.data(), sizeof(int) * et_flux.size()));
    CK(cudaStreamSynchronize(h->st));  // host vectors go out of scope
    BodyDev& b = h->body;
    b.nb = nb; b.nf = h->nf; b.nbodies = h->nbodies;
    b.xb = h->d_xb; b.ds = h->d_ds; b.bidx = h->d_bidx; b.w = h->d_w; b.body_start = h->d_body_start;
    b.n_src = (int)src_pts.size(); b.src_pts = h->d_src_pts; b.src_rows = h->d_src_rows;
    b.et_ptr = h->d_et_ptr; b.et_k = h->d_et_k; b.et_w = h->d_et_w;
    b.n_et_rows = (int)et_flux.size(); b.et_flux = h->d_et_flux;
    CK(launch_weights(g, d->h, d->offx, d->offy, b, h->st));
    return IBPM_OK;
}

// B[:, j] = E · vort2flux(A⁻¹₁ C'E' e_j)[level-1 flux] (B_times!,
// laplacian.jl:143-169), `chunk` columns per batch, then Binv = B⁻¹.
static int build_binv(ibpm_handle* h) {
    const Geom& g = h->g;
    const int nf = h->nf, mg = g.mg;
    const int chunk = std::min(nf, kBChunk);
    double *GB = nullptr, *PB = nullptr, *QB = nullptr, *work = nullptr;
    int* info = nullptr;
    int rc;
    const long long bstride = g.S * mg;
    if ((rc = dalloc(h, &GB, (size_t)bstride * chunk)) || (rc = dalloc(h, &PB, (size_t)bstride * chunk)) ||
        (rc = dalloc(h, &QB, (size_t)g.nq * chunk)) || (rc = dalloc(h, &work, gj_work_doubles(nf))) ||
        (rc = dalloc(h, &info, 1))) {
        cudaFree(GB); cudaFree(PB); cudaFree(QB); cudaFree(work); cudaFree(info);
        return rc;
    }
    // B at create is built with the single-level (latency) plan on every
    // launch, so B⁻¹, and every step it feeds, does not depend on the
    // multi-level plan chosen for the steps
    const int planN[2] = {h->px.planN, h->py.planN};
    h->px.planN = h->px.plan1;
    h->py.planN = h->py.plan1;
    auto cleanup = [&]() {
        h->px.planN = planN[0];
        h->py.planN = planN[1];
        cudaFree(GB); cudaFree(PB); cudaFree(QB); cudaFree(work); cudaFree(info);
    };
    for (int c0 = 0; c0 < nf && rc == IBPM_OK; c0 += chunk) {
        const int R = std::min(chunk, nf - c0);
        if (cudaMemsetAsync(GB, 0, sizeof(double) * bstride * R, h->st) != cudaSuccess) { rc = IBPM_ERR_CUDA; break; }
        if (launch_unit_src(g, h->body, c0, R, GB, bstride, h->st) != cudaSuccess) { rc = IBPM_ERR_CUDA; break; }
        SlabMap l0 = levmap(g, 0, 1, bstride);
        rc = poisson(h, GB, l0, GB, l0, GB, l0, R, SPEC_AINV, XEMIT_STORE);
        if (rc) break;
        rc = vort2flux(h, GB, PB, bstride, R, QB, g.nq, 0, 1);  // level-1 flux of each column
        if (rc) break;
        if (launch_E(g, h->body, QB, g.nq, R, 0.0, 0.0, h->Binv + c0, -(long long)nf, h->st) != cudaSuccess) {
            rc = IBPM_ERR_CUDA;
            break;
        }
    }
    if (rc == IBPM_OK) {
        if (launch_gj_inverse(h->Binv, nf, work, info, h->st) != cudaSuccess) rc = fail(h, IBPM_ERR_CUDA, "gj inverse launch");
    }
    int hinfo = 0;
    if (rc == IBPM_OK) {
        cudaError_t e = cudaMemcpyAsync(&hinfo, info, sizeof(int), cudaMemcpyDeviceToHost, h->st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(h->st);
        if (e != cudaSuccess) rc = fail(h, IBPM_ERR_CUDA, std::string("B setup: ") + cudaGetErrorString(e));
        else if (hinfo) rc = fail(h, IBPM_ERR_INVALID, "Schur complement B is singular (zero pivot at column " +
                                                              std::to_string(hinfo) + ")");
    }
    cleanup();
    return rc;
}

static void free_handle(ibpm_handle* h) {
    if (!h) return;
    for (int p = 0; p < 2; ++p) {
        if (h->gexec[p]) cudaGraphExecDestroy(h->gexec[p]);
        if (h->gcold[p]) cudaGraphExecDestroy(h->gcold[p]);
    }
    if (h->T32) cudaFree(h->T32);
    if (h->Pp) cudaFree(h->Pp);
    for (void* p : {(void*)h->btW, (void*)h->btU, (void*)h->btP, (void*)h->btE, (void*)h->btS, (void*)h->btY,
                    (void*)h->btY32})
        if (p) cudaFree(p);
    if (h->mtab) cudaFree(h->mtab);
    for (void* p : {(void*)h->d_x0, (void*)h->d_ub, (void*)h->d_bbox, (void*)h->btab, (void*)h->bGB, (void*)h->bPB,
                    (void*)h->bQB, (void*)h->bwork, (void*)h->binfo})
        if (p) cudaFree(p);
    if (h->GB) cudaFree(h->GB);
    if (h->qB) cudaFree(h->qB);
    for (int p = 0; p < 2; ++p) if (h->gadj[p]) cudaGraphExecDestroy(h->gadj[p]);
    void* adj[] = {h->tapeG, h->tapeq, h->ck, h->Gb, h->qb, h->Nb[0], h->Nb[1], h->Gt, h->psib, h->Wadj, h->rb,
                   h->qsb, h->Ft, h->Fbar, h->bcc, h->bcv, h->q0part, h->stepw, h->adj_n, h->wd, h->tapeFb,
                   h->tapeq1, h->gxb};
    for (void* p : adj) if (p) cudaFree(p);
    void* ptrs[] = {h->G[0], h->G[1], h->Nl[0], h->Nl[1], h->psi, h->q, h->qs, h->rhs, h->Gsrc, h->F, h->Fb,
                    h->Binv, h->nonlin1_shadow, h->d_xb, h->d_ds, h->d_bidx, h->d_w, h->d_body_start,
                    h->d_src_pts, h->d_src_rows, h->d_et_ptr, h->d_et_k, h->d_et_w, h->d_et_flux, h->hist,
                    h->counter, h->status};
    for (void* p : ptrs) if (p) cudaFree(p);
    if (h->flush_buf) cudaFree(h->flush_buf);
    if (h->pin_hist) cudaFreeHost(h->pin_hist);
    if (h->pin_status) cudaFreeHost(h->pin_status);
    for (cudaEvent_t e : h->prof_ev) cudaEventDestroy(e);
    if (h->have_px) dst_plan_destroy(&h->px);
    if (h->have_py) dst_plan_destroy(&h->py);
    if (h->st) cudaStreamDestroy(h->st);
    delete h;
}

// ---------------------------------------------------------------------------
// Public API
// ---------------------------------------------------------------------------
extern "C" const char* ibpm_version(void) { return IBPM_VERSION_STR; }

extern "C" const char* ibpm_last_error(const ibpm_handle* h) {
    return h ? h->err.c_str() : g_create_err.c_str();
}

static int create_impl(ibpm_handle* h, const ibpm_problem_desc* d) {
    if (d->nx < 8 || d->ny < 8 || d->nx % 4 || d->ny % 4)
        return fail(h, IBPM_ERR_INVALID, "nx and ny must be multiples of 4 and at least 8");
    if (d->mg < 1 || d->mg > 8) return fail(h, IBPM_ERR_INVALID, "mg must be in 1..8");
    if (!(d->h > 0) || !(d->dt > 0) || !(d->Re > 0)) return fail(h, IBPM_ERR_INVALID, "h, dt and Re must be positive");
    if (d->nb < 1 || d->nbodies < 1 || !d->xb || !d->ds || !d->body_npts)
        return fail(h, IBPM_ERR_INVALID, "at least one body with one point is required");
    if (d->precision != IBPM_PREC_FP64 && d->precision != IBPM_PREC_FP32_REFINED)
        return fail(h, IBPM_ERR_INVALID, "precision must be IBPM_PREC_FP64 or IBPM_PREC_FP32_REFINED");
    if (d->refine_sweeps < 0 || d->refine_sweeps > 8) return fail(h, IBPM_ERR_INVALID, "refine_sweeps must be in 0..8");
    h->prec = d->precision;
    h->sweeps = std::max(1, (int)d->refine_sweeps);
    int tot = 0;
    for (int j = 0; j < d->nbodies; ++j) {
        if (d->body_npts[j] < 1) return fail(h, IBPM_ERR_INVALID, "every body needs at least one point");
        tot += d->body_npts[j];
    }
    if (tot != d->nb) return fail(h, IBPM_ERR_INVALID, "sum(body_npts) != nb");
    h->device = d->device;
    CK(cudaSetDevice(d->device));
    CK(cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking));
    h->g = make_geom(d->nx, d->ny, d->mg);
    h->h = d->h; h->offx = d->offx; h->offy = d->offy; h->Re = d->Re; h->dt = d->dt;
    h->Ux = d->Ux; h->Uy = d->Uy; h->incl = d->inclination;
    h->beta[0] = d->beta[0]; h->beta[1] = d->beta[1];
    h->nb = d->nb; h->nf = 2 * d->nb; h->nbodies = d->nbodies;
    h->body_start.assign(d->nbodies + 1, 0);
    for (int j = 0; j < d->nbodies; ++j) h->body_start[j + 1] = h->body_start[j] + d->body_npts[j];
    const Geom& g = h->g;
    const char* sup = "32, 64, 128, 192, 200, 256, 384, 400, 512, 768, 1024, 2048";
    if (!dst_supported(g.nx)) return fail(h, IBPM_ERR_UNSUPPORTED, std::string("nx must be one of ") + sup);
    if (!dst_supported(g.ny)) return fail(h, IBPM_ERR_UNSUPPORTED, std::string("ny must be one of ") + sup);
    if (dst_plan_create(&h->px, g.nx, h->st)) return fail(h, IBPM_ERR_CUDA, "DST plan (x) setup failed");
    h->have_px = true;
    if (dst_plan_create(&h->py, g.ny, h->st)) return fail(h, IBPM_ERR_CUDA, "DST plan (y) setup failed");
    h->have_py = true;
    // base_flux! for inertial motion (timestepping.jl:252-270)
    for (int l = 0; l < g.mg; ++l) {
        const double hc = d->h * std::ldexp(1.0, l);
        const double a = d->inclination;
        h->q0x[l] = (d->Ux * std::cos(a) - d->Uy * std::sin(a)) * hc;
        h->q0y[l] = (d->Ux * std::sin(a) + d->Uy * std::cos(a)) * hc;
    }
    const size_t slabs = (size_t)g.S * g.mg;
    int rc;
    if ((rc = dalloc(h, &h->G[0], slabs)) || (rc = dalloc(h, &h->G[1], slabs)) || (rc = dalloc(h, &h->Nl[0], slabs)) ||
        (rc = dalloc(h, &h->Nl[1], slabs)) || (rc = dalloc(h, &h->psi, slabs)) ||
        (rc = dalloc(h, &h->q, (size_t)g.nq * g.mg)) || (rc = dalloc(h, &h->qs, (size_t)g.nq * g.mg)) ||
        (rc = dalloc(h, &h->rhs, slabs)) || (rc = dalloc(h, &h->Gsrc, g.S)) || (rc = dalloc(h, &h->F, h->nf)) ||
        (rc = dalloc(h, &h->Fb, h->nf)) || (rc = dalloc(h, &h->Binv, (size_t)h->nf * h->nf)) ||
        (rc = dalloc(h, &h->nonlin1_shadow, slabs)) || (rc = dalloc(h, &h->counter, 1)) ||
        (rc = dalloc(h, &h->status, 1)))
        return rc;
    for (double* p : {h->G[0], h->G[1], h->Nl[0], h->Nl[1], h->psi, h->rhs, h->nonlin1_shadow})
        CK(cudaMemsetAsync(p, 0, sizeof(double) * slabs, h->st));
    CK(cudaMemsetAsync(h->q, 0, sizeof(double) * g.nq * g.mg, h->st));
    CK(cudaMemsetAsync(h->qs, 0, sizeof(double) * g.nq * g.mg, h->st));
    CK(cudaMemsetAsync(h->Gsrc, 0, sizeof(double) * g.S, h->st));
    CK(cudaMemsetAsync(h->Fb, 0, sizeof(double) * h->nf, h->st));
    CK(cudaMemsetAsync(h->status, 0, sizeof(int), h->st));
    if (h->prec == IBPM_PREC_FP32_REFINED) {
        if ((rc = dalloc(h, &h->T32, slabs)) || (rc = dalloc(h, &h->Pp, g.S))) return rc;
        CK(cudaMemsetAsync(h->T32, 0, sizeof(float) * slabs, h->st));
        CK(cudaMemsetAsync(h->Pp, 0, sizeof(double) * g.S, h->st));
    }
    if ((rc = build_coupling(h, d))) return rc;
    if ((rc = build_binv(h))) return rc;
    // the boundary-transfer level chain where its factors exist
    if ((rc = build_bt(h))) return rc;
    if (g.mg >= 2 && !h->bt) h->chain = IBPM_CHAIN_SEQUENTIAL;
    CK(cudaStreamSynchronize(h->st));
    return IBPM_OK;
}

extern "C" int ibpm_create(const ibpm_problem_desc* desc, ibpm_handle** out) {
    if (!desc || !out) {
        g_create_err = "null argument";
        return IBPM_ERR_INVALID;
    }
    *out = nullptr;
    ibpm_handle* h = new ibpm_handle();
    int rc = create_impl(h, desc);
    if (rc != IBPM_OK) {
        g_create_err = h->err;
        free_handle(h);
        return rc;
    }
    g_create_err.clear();
    *out = h;
    return IBPM_OK;
}

extern "C" int ibpm_destroy(ibpm_handle* h) {
    if (!h) return IBPM_ERR_INVALID;
    if (h->in_batch) return fail(h, IBPM_ERR_INVALID, "a batch member is released with its batch (ibpm_batch_destroy)");
    cudaSetDevice(h->device);
    cudaStreamSynchronize(h->st);
    free_handle(h);
    return IBPM_OK;
}

extern "C" int ibpm_sizes(const ibpm_handle* h, int64_t* nGamma, int64_t* nq, int32_t* mg, int32_t* nf,
                          int32_t* nbodies) {
    if (!h) return IBPM_ERR_INVALID;
    if (nGamma) *nGamma = (int64_t)h->g.n1 * h->g.n2;
    if (nq) *nq = h->g.nq;
    if (mg) *mg = h->g.mg;
    if (nf) *nf = h->nf;
    if (nbodies) *nbodies = h->nbodies;
    return IBPM_OK;
}

// Γ-like (nΓ, mg) column-major host matrix <-> padded device slabs: the rows
// of all levels are consecutive on both sides, so one 2-D copy moves them.
static cudaError_t slab_copy(ibpm_handle* h, double* dst, const double* src, bool to_device) {
    const Geom& g = h->g;
    const size_t w = sizeof(double) * g.n1, rows = (size_t)g.n2 * g.mg;
    if (to_device) return cudaMemcpy2DAsync(dst, sizeof(double) * g.P, src, w, w, rows, cudaMemcpyHostToDevice, h->st);
    return cudaMemcpy2DAsync(dst, w, src, sizeof(double) * g.P, w, rows, cudaMemcpyDeviceToHost, h->st);
}

extern "C" int ibpm_set_state(ibpm_handle* h, const double* Gamma, const double* q, const double* q0,
                              const double* psi, const double* nonlin1, const double* nonlin2, const double* Fb) {
    if (!h) return IBPM_ERR_INVALID;
    CK(cudaSetDevice(h->device));
    const Geom& g = h->g;
    if (q0 && !h->moving) {  // a moving grid's q0 is recomputed at every step (timestepping.jl:41-43)
        double nx0[8], ny0[8];
        for (int l = 0; l < g.mg; ++l) {
            const double* ql = q0 + (size_t)l * g.nq;
            nx0[l] = ql[0];
            ny0[l] = ql[g.nu];
            for (int e = 0; e < g.nu; ++e)
                if (ql[e] != nx0[l]) return fail(h, IBPM_ERR_UNSUPPORTED, "q0 must be uniform per level (x part)");
            for (int e = g.nu; e < g.nq; ++e)
                if (ql[e] != ny0[l]) return fail(h, IBPM_ERR_UNSUPPORTED, "q0 must be uniform per level (y part)");
        }
        bool changed = false;
        for (int l = 0; l < g.mg; ++l) {
            changed |= h->q0x[l] != nx0[l] || h->q0y[l] != ny0[l];
            h->q0x[l] = nx0[l]; h->q0y[l] = ny0[l];
        }
        if (changed) {  // q0 is baked into the captured step and its adjoint
            h->graphs_ready = false;
            for (int p = 0; p < 2; ++p) if (h->gadj[p]) { cudaGraphExecDestroy(h->gadj[p]); h->gadj[p] = nullptr; }
        }
    }
    if (Gamma) CK(slab_copy(h, h->G[h->cur], Gamma, true));
    if (psi) CK(slab_copy(h, h->psi, psi, true));
    if (q) CK(cudaMemcpyAsync(h->q, q, sizeof(double) * g.nq * g.mg, cudaMemcpyHostToDevice, h->st));
    if (nonlin2) CK(slab_copy(h, h->Nl[h->cur], nonlin2, true));
    if (nonlin1) {
        CK(slab_copy(h, h->nonlin1_shadow, nonlin1, true));
        h->nonlin1_valid = true;
    }
    if (Fb) CK(cudaMemcpyAsync(h->Fb, Fb, sizeof(double) * h->nf, cudaMemcpyHostToDevice, h->st));
    CK(cudaStreamSynchronize(h->st));
    if (Gamma || psi) {
        // the refined mode's hidden initial guess of the projection solve is
        // cleared, so results depend only on the state given (ψ is the other
        // guess; it is part of the state)
        h->cold = kColdSteps;
        if (h->Pp) CK(cudaMemsetAsync(h->Pp, 0, sizeof(double) * g.S, h->st));
        CK(cudaStreamSynchronize(h->st));
    }
    return IBPM_OK;
}

extern "C" int ibpm_set_base_state(ibpm_handle* h, const double* Gamma_B, const double* q_B) {
    if (!h || !Gamma_B || !q_B) return IBPM_ERR_INVALID;
    CK(cudaSetDevice(h->device));
    const Geom& g = h->g;
    const size_t slabs = (size_t)g.S * g.mg;
    if (!h->GB) {
        int rc;
        if ((rc = dalloc(h, &h->GB, slabs)) || (rc = dalloc(h, &h->qB, (size_t)g.nq * g.mg))) return rc;
        CK(cudaMemsetAsync(h->GB, 0, sizeof(double) * slabs, h->st));
    }
    CK(slab_copy(h, h->GB, Gamma_B, true));
    CK(cudaMemcpyAsync(h->qB, q_B, sizeof(double) * g.nq * g.mg, cudaMemcpyHostToDevice, h->st));
    if (!h->lin) {
        // the base state carries the problem's base flux; the perturbation's is
        // zero (base_flux! of a LinearizedIBProblem, timestepping.jl:236-250)
        for (int l = 0; l < g.mg; ++l) {
            h->q0Bx[l] = h->q0x[l]; h->q0By[l] = h->q0y[l];
            h->q0x[l] = 0.0; h->q0y[l] = 0.0;
        }
        h->lin = true;
    }
    h->graphs_ready = false;
    for (int p = 0; p < 2; ++p) if (h->gadj[p]) { cudaGraphExecDestroy(h->gadj[p]); h->gadj[p] = nullptr; }
    h->cold = kColdSteps;
    CK(cudaStreamSynchronize(h->st));
    return IBPM_OK;
}

extern "C" int ibpm_get_state(ibpm_handle* h, double* Gamma, double* q, double* q0, double* psi, double* nonlin1,
                              double* nonlin2, double* Fb) {
    if (!h) return IBPM_ERR_INVALID;
    CK(cudaSetDevice(h->device));
    const Geom& g = h->g;
    if (Gamma) CK(slab_copy(h, Gamma, h->G[h->cur], false));
    if (psi) CK(slab_copy(h, psi, h->psi, false));
    if (q) CK(cudaMemcpyAsync(q, h->q, sizeof(double) * g.nq * g.mg, cudaMemcpyDeviceToHost, h->st));
    if (nonlin2) CK(slab_copy(h, nonlin2, h->Nl[h->cur], false));
    if (nonlin1) CK(slab_copy(h, nonlin1, h->nonlin1_valid ? h->nonlin1_shadow : h->Nl[h->cur], false));
    if (Fb) CK(cudaMemcpyAsync(Fb, h->Fb, sizeof(double) * h->nf, cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    if (q0 && h->moving) {
        // the base flux of the last step's motion row, by the device's formula
        const double* r = h->mv_last;
        for (int l = 0; l < g.mg; ++l) {
            const double hc = h->h * std::ldexp(1.0, l);
            double* ql = q0 + (size_t)l * g.nq;
            for (int j = 1; j <= g.ny; ++j) {
                const double y = (((j - 0.5) - 0.5 * g.ny) * hc + (0.5 * g.ny) * h->h) - h->offy;
                const double v = (y - h->mv_yc) * (-hc * r[0]) + hc * r[1];
                for (int i = 0; i <= g.nx; ++i) ql[i + (size_t)(j - 1) * (g.nx + 1)] = v;
            }
            for (int i = 1; i <= g.nx; ++i) {
                const double x = (((i - 0.5) - 0.5 * g.nx) * hc + (0.5 * g.nx) * h->h) - h->offx;
                const double v = (x - h->mv_xc) * (hc * r[0]) + hc * r[2];
                for (int j = 0; j <= g.ny; ++j) ql[g.nu + (i - 1) + (size_t)j * g.nx] = v;
            }
        }
    } else if (q0) {
        for (int l = 0; l < g.mg; ++l) {
            double* ql = q0 + (size_t)l * g.nq;
            for (int e = 0; e < g.nu; ++e) ql[e] = h->q0x[l];
            for (int e = g.nu; e < g.nq; ++e) ql[e] = h->q0y[l];
        }
    }
    return IBPM_OK;
}

extern "C" int ibpm_set_moving_grid(ibpm_handle* h, double xc, double yc, const double* motion0) {
    if (!h || !motion0) return IBPM_ERR_INVALID;
    if (h->nbodies != 1) return fail(h, IBPM_ERR_UNSUPPORTED, "a moving grid carries exactly one body");
    if (h->lin) return fail(h, IBPM_ERR_UNSUPPORTED, "a linearised problem has no moving-grid base flux");
    if (h->bodies_moving) return fail(h, IBPM_ERR_UNSUPPORTED, "the bodies already move (MotionFunction)");
    if (!std::isfinite(xc) || !std::isfinite(yc)) return fail(h, IBPM_ERR_INVALID, "xc and yc must be finite");
    CK(cudaSetDevice(h->device));
    CK(cudaStreamSynchronize(h->st));
    h->moving = true;
    h->mv_xc = xc; h->mv_yc = yc;
    moving_rates(h, motion0, h->mv_last);
    h->graphs_ready = false;  // the step now reads the per-step rows
    for (int p = 0; p < 2; ++p) if (h->gadj[p]) { cudaGraphExecDestroy(h->gadj[p]); h->gadj[p] = nullptr; }
    return IBPM_OK;
}

static int ensure_graphs(ibpm_handle* h, int cap) {
    if (h->graphs_ready && h->hist_cap >= cap) return IBPM_OK;
    if (h->hist_cap < cap) {
        if (h->hist) cudaFree(h->hist);
        h->hist = nullptr;
        int rc = dalloc(h, &h->hist, (size_t)cap * 2 * h->nbodies);
        if (rc) return rc;
        if (h->pin_hist) cudaFreeHost(h->pin_hist);
        h->pin_hist = nullptr;
        if (cudaMallocHost((void**)&h->pin_hist, sizeof(double) * cap * 2 * h->nbodies) != cudaSuccess) {
            h->pin_hist = nullptr;
            return fail(h, IBPM_ERR_NOMEM, "cudaMallocHost: force history mirror");
        }
        h->hist_cap = cap;
    }
    if (!h->pin_status && cudaMallocHost((void**)&h->pin_status, sizeof(int)) != cudaSuccess) {
        h->pin_status = nullptr;
        return fail(h, IBPM_ERR_NOMEM, "cudaMallocHost: status word");
    }
    if (h->bodies_moving && h->btab_cap < h->hist_cap) {
        if (h->btab) cudaFree(h->btab);
        h->btab = nullptr;
        h->btab_cap = 0;
        int rc = dalloc(h, &h->btab, (size_t)h->hist_cap * h->nbodies * 8);
        if (rc) return rc;
        CK(cudaMemsetAsync(h->btab, 0, sizeof(double) * h->hist_cap * h->nbodies * 8, h->st));
        h->btab_cap = h->hist_cap;
    }
    if (h->moving && h->mtab_cap < h->hist_cap) {
        if (h->mtab) cudaFree(h->mtab);
        h->mtab = nullptr;
        h->mtab_cap = 0;
        int rc = dalloc(h, &h->mtab, (size_t)h->hist_cap * 3);
        if (rc) return rc;
        CK(cudaMemsetAsync(h->mtab, 0, sizeof(double) * 3 * h->hist_cap, h->st));
        h->mtab_cap = h->hist_cap;
    }
    const int nkind = h->prec == IBPM_PREC_FP32_REFINED ? 2 : 1;
    for (int kind = 0; kind < nkind; ++kind)
        for (int p = 0; p < 2; ++p) {
            cudaGraphExec_t& ge = kind ? h->gcold[p] : h->gexec[p];
            if (ge) { cudaGraphExecDestroy(ge); ge = nullptr; }
            cudaGraph_t graph;
            CK(cudaStreamBeginCapture(h->st, cudaStreamCaptureModeThreadLocal));
            int rc = enqueue_step(h, p, kind == 1);
            cudaError_t e = cudaStreamEndCapture(h->st, &graph);
            if (rc) return rc;
            if (e != cudaSuccess) return fail(h, IBPM_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
            e = cudaGraphInstantiate(&ge, graph, 0);
            cudaGraphDestroy(graph);
            if (e != cudaSuccess)
                return fail(h, IBPM_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
        }
    h->graphs_ready = true;
    return IBPM_OK;
}

// Queue one step from the current parity.  In FP32_REFINED mode the first
// kColdSteps steps after create or set_state run one more correction sweep
// per solve (see kColdSteps).
static cudaError_t launch_step(ibpm_handle* h) {
    cudaGraphExec_t ge = (h->cold > 0 && h->gcold[h->cur]) ? h->gcold[h->cur] : h->gexec[h->cur];
    if (h->cold > 0) --h->cold;
    const cudaError_t e = cudaGraphLaunch(ge, h->st);
    h->cur ^= 1;
    return e;
}

// Steps of ibpm_advance, ibpm_advance_moving and ibpm_advance_bodies;
// `motion` holds each step's U, V, θ, θ̇ (moving grid) or, per body, x, y, θ,
// ẋ, ẏ, θ̇ (moving bodies).
static int advance_impl(ibpm_handle* h, int32_t nsteps, const double* motion, double* CD_out, double* CL_out) {
    if (nsteps == 0) return IBPM_OK;
    CK(cudaSetDevice(h->device));
    const int cap = std::max(1024, std::min(nsteps, 4096));
    int rc = ensure_graphs(h, std::max(cap, h->hist_cap));
    if (rc) return rc;
    CK(cudaMemsetAsync(h->status, 0, sizeof(int), h->st));
    int done = 0;
    while (done < nsteps) {
        const int n = std::min(h->hist_cap, nsteps - done);
        if (motion && h->bodies_moving) {
            // (x, y, cos θ, sin θ, ẋ, ẏ, θ̇, 0) per body and step (TangentSE2, move-body-utils.jl:70-84)
            std::vector<double> rows((size_t)8 * n * h->nbodies);
            for (int s = 0; s < n; ++s)
                for (int j = 0; j < h->nbodies; ++j) {
                    const double* m = motion + 6 * ((size_t)(done + s) * h->nbodies + j);
                    double* r = &rows[8 * ((size_t)s * h->nbodies + j)];
                    r[0] = m[0]; r[1] = m[1]; r[2] = std::cos(m[2]); r[3] = std::sin(m[2]);
                    r[4] = m[3]; r[5] = m[4]; r[6] = m[5]; r[7] = 0.0;
                }
            CK(cudaMemcpyAsync(h->btab, rows.data(), sizeof(double) * rows.size(), cudaMemcpyHostToDevice, h->st));
            CK(cudaStreamSynchronize(h->st));
        } else if (motion) {
            // this chunk's rows; the copy is ordered after the previous chunk's steps
            std::vector<double> rows((size_t)3 * n);
            for (int s = 0; s < n; ++s) moving_rates(h, motion + 4 * (size_t)(done + s), &rows[3 * (size_t)s]);
            CK(cudaMemcpyAsync(h->mtab, rows.data(), sizeof(double) * rows.size(), cudaMemcpyHostToDevice, h->st));
            CK(cudaStreamSynchronize(h->st));
            std::copy(rows.end() - 3, rows.end(), h->mv_last);
        }
        CK(cudaMemsetAsync(h->counter, 0, sizeof(int), h->st));
        for (int s = 0; s < n; ++s) CK(launch_step(h));
        h->nonlin1_valid = false;
        // the chunk's CD/CL (and after the last chunk the status word) into
        // page-locked memory, one synchronisation for both
        const bool last = done + n >= nsteps;
        if (CD_out || CL_out)
            CK(cudaMemcpyAsync(h->pin_hist, h->hist, sizeof(double) * n * 2 * h->nbodies, cudaMemcpyDeviceToHost,
                               h->st));
        if (last) CK(cudaMemcpyAsync(h->pin_status, h->status, sizeof(int), cudaMemcpyDeviceToHost, h->st));
        if (CD_out || CL_out || last) CK(cudaStreamSynchronize(h->st));
        if (CD_out || CL_out) {
            const double* hb = h->pin_hist;
            for (int s = 0; s < n; ++s)
                for (int j = 0; j < h->nbodies; ++j) {
                    if (CD_out) CD_out[(size_t)(done + s) * h->nbodies + j] = hb[((size_t)s * 2 + 0) * h->nbodies + j];
                    if (CL_out) CL_out[(size_t)(done + s) * h->nbodies + j] = hb[((size_t)s * 2 + 1) * h->nbodies + j];
                }
        }
        done += n;
    }
    const int hstatus = *h->pin_status;
    if (hstatus & 8) return fail(h, IBPM_ERR_CUDA, "internal: a step ran past the force history");
    if (hstatus & 4) return fail(h, IBPM_ERR_INVALID, "a moving body's regularisation stencil left the finest grid");
    if (hstatus & 2) return fail(h, IBPM_ERR_NONFINITE, "the Schur complement B of the moved bodies is singular");
    if (hstatus) return fail(h, IBPM_ERR_NONFINITE, "CD/CL became non-finite");
    return IBPM_OK;
}

extern "C" int ibpm_advance(ibpm_handle* h, double t, int32_t nsteps, double* CD_out, double* CL_out) {
    (void)t;
    if (!h || nsteps < 0) return IBPM_ERR_INVALID;
    if (h->moving) return fail(h, IBPM_ERR_INVALID, "a moving grid needs each step's motion: use ibpm_advance_moving");
    if (h->bodies_moving)
        return fail(h, IBPM_ERR_INVALID, "moving bodies need each step's motion: use ibpm_advance_bodies");
    return advance_impl(h, nsteps, nullptr, CD_out, CL_out);
}

extern "C" int ibpm_set_motion_function(ibpm_handle* h) {
    if (!h) return IBPM_ERR_INVALID;
    if (h->lin) return fail(h, IBPM_ERR_UNSUPPORTED, "a linearised problem has fixed bodies");
    if (h->moving) return fail(h, IBPM_ERR_UNSUPPORTED, "the grid already moves with the body (MovingGrid)");
    if (h->bodies_moving) return IBPM_OK;
    CK(cudaSetDevice(h->device));
    const Geom& g = h->g;
    const int nf = h->nf, chunk = std::min(nf, kBChunk);
    const long long bstride = g.S * g.mg;
    int rc;
    if ((rc = dalloc(h, &h->d_x0, 2 * h->nb)) || (rc = dalloc(h, &h->d_ub, 2 * h->nb)) ||
        (rc = dalloc(h, &h->d_bbox, 4)) || (rc = dalloc(h, &h->bGB, (size_t)bstride * chunk)) ||
        (rc = dalloc(h, &h->bPB, (size_t)bstride * chunk)) || (rc = dalloc(h, &h->bQB, (size_t)g.nq * chunk)) ||
        (rc = dalloc(h, &h->bwork, gj_work_doubles(nf))) || (rc = dalloc(h, &h->binfo, 1)))
        return rc;
    // the reference configuration x0 is the body as created (RigidBody.x0)
    CK(cudaMemcpyAsync(h->d_x0, h->d_xb, sizeof(double) * 2 * h->nb, cudaMemcpyDeviceToDevice, h->st));
    CK(cudaMemsetAsync(h->d_ub, 0, sizeof(double) * 2 * h->nb, h->st));
    CK(cudaStreamSynchronize(h->st));
    h->bodies_moving = true;
    h->graphs_ready = false;
    for (int p = 0; p < 2; ++p) if (h->gadj[p]) { cudaGraphExecDestroy(h->gadj[p]); h->gadj[p] = nullptr; }
    return IBPM_OK;
}

extern "C" int ibpm_advance_bodies(ibpm_handle* h, int32_t nsteps, const double* motion, double* CD_out,
                                   double* CL_out) {
    if (!h || nsteps < 0 || (nsteps > 0 && !motion)) return IBPM_ERR_INVALID;
    if (!h->bodies_moving) return fail(h, IBPM_ERR_INVALID, "bodies are fixed: call ibpm_set_motion_function first");
    for (int64_t e = 0; e < 6 * (int64_t)nsteps * h->nbodies; ++e)
        if (!std::isfinite(motion[e])) return fail(h, IBPM_ERR_INVALID, "motion values must be finite");
    return advance_impl(h, nsteps, motion, CD_out, CL_out);
}

extern "C" int ibpm_get_body_points(ibpm_handle* h, double* xb, double* ub) {
    if (!h) return IBPM_ERR_INVALID;
    CK(cudaSetDevice(h->device));
    if (xb) CK(cudaMemcpyAsync(xb, h->d_xb, sizeof(double) * 2 * h->nb, cudaMemcpyDeviceToHost, h->st));
    if (ub) {
        if (h->bodies_moving) CK(cudaMemcpyAsync(ub, h->d_ub, sizeof(double) * 2 * h->nb, cudaMemcpyDeviceToHost, h->st));
        else std::fill(ub, ub + 2 * h->nb, 0.0);
    }
    CK(cudaStreamSynchronize(h->st));
    return IBPM_OK;
}

extern "C" int ibpm_advance_moving(ibpm_handle* h, int32_t nsteps, const double* motion, double* CD_out,
                                   double* CL_out) {
    if (!h || nsteps < 0 || (nsteps > 0 && !motion)) return IBPM_ERR_INVALID;
    if (!h->moving) return fail(h, IBPM_ERR_INVALID, "not a moving grid: call ibpm_set_moving_grid first");
    for (int64_t e = 0; e < 4 * (int64_t)nsteps; ++e)
        if (!std::isfinite(motion[e])) return fail(h, IBPM_ERR_INVALID, "motion values must be finite");
    return advance_impl(h, nsteps, motion, CD_out, CL_out);
}

extern "C" int ibpm_vort2flux(ibpm_handle* h) {
    if (!h) return IBPM_ERR_INVALID;
    CK(cudaSetDevice(h->device));
    int rc = h->bt ? vort2flux_bt(h, h->G[h->cur], h->q, h->g.mg, h->g.mg)
                   : vort2flux(h, h->G[h->cur], h->psi, h->g.S * h->g.mg, 1, h->q, 0, 0, h->g.mg);
    if (rc) return rc;
    CK(cudaStreamSynchronize(h->st));
    return IBPM_OK;
}

extern "C" int ibpm_get_binv(ibpm_handle* h, double* Binv) {
    if (!h || !Binv) return IBPM_ERR_INVALID;
    CK(cudaSetDevice(h->device));
    const int nf = h->nf;
    std::vector<double> rm((size_t)nf * nf);
    CK(cudaMemcpyAsync(rm.data(), h->Binv, sizeof(double) * rm.size(), cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    for (int i = 0; i < nf; ++i)
        for (int j = 0; j < nf; ++j) Binv[(size_t)i + (size_t)j * nf] = rm[(size_t)i * nf + j];
    return IBPM_OK;
}

// Transform plan of the handle's sine transforms: the latency plan (radix 4,
// the default for single-slab launches) or the throughput plan (radix 8).
// The step graphs are captured again on the next advance.
static void set_plans(ibpm_handle* h, int single_slab, int multi_slab) {
    for (DstPlan* p : {&h->px, &h->py}) {
        p->plan1 = single_slab;
        p->planN = multi_slab;
    }
    h->graphs_ready = false;
    for (int p = 0; p < 2; ++p) if (h->gadj[p]) { cudaGraphExecDestroy(h->gadj[p]); h->gadj[p] = nullptr; }
}

extern "C" int ibpm_set_transform_plan(ibpm_handle* h, int32_t single_slab, int32_t multi_slab) {
    if (!h) return IBPM_ERR_INVALID;
    if (single_slab != IBPM_PLAN_LATENCY && single_slab != IBPM_PLAN_THROUGHPUT)
        return fail(h, IBPM_ERR_INVALID, "single-slab plan must be IBPM_PLAN_LATENCY or IBPM_PLAN_THROUGHPUT");
    if (multi_slab != IBPM_PLAN_LATENCY && multi_slab != IBPM_PLAN_THROUGHPUT && multi_slab != IBPM_PLAN_AUTO)
        return fail(h, IBPM_ERR_INVALID,
                    "multi-slab plan must be IBPM_PLAN_LATENCY, IBPM_PLAN_THROUGHPUT or IBPM_PLAN_AUTO");
    CK(cudaSetDevice(h->device));
    CK(cudaStreamSynchronize(h->st));
    set_plans(h, single_slab, multi_slab);
    return IBPM_OK;
}

// The level chain of vort2flux!: the boundary transfer builds its factors on
// first use; a single level has no chain, and either setting is kept.
static int set_chain(ibpm_handle* h, int chain) {
    const bool want = chain == IBPM_CHAIN_BOUNDARY_TRANSFER && h->g.mg >= 2, was = h->bt;
    if (want && !h->btW) {
        int rc = build_bt(h);
        if (rc) return rc;
        if (!h->btW)
            return fail(h, IBPM_ERR_UNSUPPORTED, "boundary transfer: the edge operator of this grid has no "
                                                 "low-rank factors (numerical rank 1024 or more)");
    }
    h->chain = chain;
    h->bt = want;
    if (want != was) {
        h->graphs_ready = false;
        for (int p = 0; p < 2; ++p) if (h->gadj[p]) { cudaGraphExecDestroy(h->gadj[p]); h->gadj[p] = nullptr; }
    }
    return IBPM_OK;
}

extern "C" int ibpm_set_level_chain(ibpm_handle* h, int32_t chain) {
    if (!h) return IBPM_ERR_INVALID;
    if (chain != IBPM_CHAIN_SEQUENTIAL && chain != IBPM_CHAIN_BOUNDARY_TRANSFER)
        return fail(h, IBPM_ERR_INVALID, "level chain must be IBPM_CHAIN_SEQUENTIAL or IBPM_CHAIN_BOUNDARY_TRANSFER");
    CK(cudaSetDevice(h->device));
    CK(cudaStreamSynchronize(h->st));
    return set_chain(h, chain);
}

extern "C" int ibpm_get_level_chain(const ibpm_handle* h, int32_t* chain) {
    if (!h || !chain) return IBPM_ERR_INVALID;
    *chain = h->chain;
    return IBPM_OK;
}

extern "C" int ibpm_get_transform_plan(const ibpm_handle* h, int32_t* single_slab, int32_t* multi_slab) {
    if (!h || !single_slab || !multi_slab) return IBPM_ERR_INVALID;
    *single_slab = h->px.plan1;
    *multi_slab = h->px.planN;
    return IBPM_OK;
}

extern "C" int ibpm_sync(ibpm_handle* h) {
    if (!h) return IBPM_ERR_INVALID;
    CK(cudaSetDevice(h->device));
    CK(cudaStreamSynchronize(h->st));
    return IBPM_OK;
}

extern "C" int ibpm_launches_per_step(ibpm_handle* h) {
    if (!h) return IBPM_ERR_INVALID;
    int rc = ensure_graphs(h, std::max(1024, h->hist_cap));
    if (rc) return rc;
    const int before = h->launches;
    cudaGraph_t graph;
    CK(cudaStreamBeginCapture(h->st, cudaStreamCaptureModeThreadLocal));
    rc = enqueue_step(h, h->cur);
    cudaError_t e = cudaStreamEndCapture(h->st, &graph);
    if (e == cudaSuccess) cudaGraphDestroy(graph);
    if (rc) return rc;
    return h->launches - before;
}

extern "C" int ibpm_bench(ibpm_handle* h, int32_t nsteps, int32_t flush_l2, double* step_ms) {
    if (!h || nsteps < 1 || !step_ms) return IBPM_ERR_INVALID;
    CK(cudaSetDevice(h->device));
    int rc = ensure_graphs(h, std::max(1024, h->hist_cap));
    if (rc) return rc;
    if (flush_l2 && !h->flush_buf) {
        h->flush_bytes = (size_t)512 << 20;  // 4x the 126 MB L2
        if ((rc = dalloc(h, (char**)&h->flush_buf, h->flush_bytes))) return rc;
    }
    std::vector<cudaEvent_t> ev(2 * nsteps);
    for (auto& e : ev) CK(cudaEventCreate(&e));
    int done = 0;
    while (done < nsteps) {
        const int n = std::min(h->hist_cap, nsteps - done);
        CK(cudaMemsetAsync(h->counter, 0, sizeof(int), h->st));
        for (int s = 0; s < n; ++s) {
            if (flush_l2) CK(cudaMemsetAsync(h->flush_buf, (done + s) & 0xff, h->flush_bytes, h->st));
            CK(cudaEventRecord(ev[2 * (done + s)], h->st));
            CK(launch_step(h));
            CK(cudaEventRecord(ev[2 * (done + s) + 1], h->st));
        }
        done += n;
    }
    h->nonlin1_valid = false;
    CK(cudaStreamSynchronize(h->st));
    for (int s = 0; s < nsteps; ++s) {
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, ev[2 * s], ev[2 * s + 1]));
        step_ms[s] = ms;
    }
    for (auto& e : ev) cudaEventDestroy(e);
    return IBPM_OK;
}

extern "C" int ibpm_profile(ibpm_handle* h, int32_t nsteps, int32_t flush_l2, double* ms_out,
                            double* bytes_out, int32_t* calls_out) {
    if (!h || nsteps < 1 || !ms_out || !bytes_out || !calls_out) return IBPM_ERR_INVALID;
    CK(cudaSetDevice(h->device));
    if (flush_l2 && !h->flush_buf) {
        h->flush_bytes = (size_t)512 << 20;
        int rc = dalloc(h, (char**)&h->flush_buf, h->flush_bytes);
        if (rc) return rc;
    }
    int rc = ensure_graphs(h, std::max(1024, h->hist_cap));
    if (rc) return rc;
    for (int k = 0; k < K_COUNT; ++k) { ms_out[k] = 0; bytes_out[k] = 0; calls_out[k] = 0; }
    // Capture one step of each parity with an event pair around every launch:
    // the replays give each kernel's device time in graph context.
    while ((int)h->prof_ev.size() < 512) {
        cudaEvent_t e;
        CK(cudaEventCreate(&e));
        h->prof_ev.push_back(e);
    }
    cudaGraphExec_t pexec[2] = {nullptr, nullptr};
    std::vector<int> lab[2];
    std::vector<double> byt[2];
    int nlaunch[2] = {0, 0};
    for (int p = 0; p < 2 && rc == IBPM_OK; ++p) {
        h->prof_on = true;
        h->prof_n = 0;
        h->prof_lab.clear();
        h->prof_bytes.clear();
        cudaGraph_t graph;
        CK(cudaStreamBeginCapture(h->st, cudaStreamCaptureModeThreadLocal));
        rc = enqueue_step(h, p);
        cudaError_t e = cudaStreamEndCapture(h->st, &graph);
        h->prof_on = false;
        if (rc) break;
        if (e != cudaSuccess) { rc = fail(h, IBPM_ERR_CUDA, cudaGetErrorString(e)); break; }
        e = cudaGraphInstantiate(&pexec[p], graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) { rc = fail(h, IBPM_ERR_CUDA, cudaGetErrorString(e)); break; }
        lab[p] = h->prof_lab;
        byt[p] = h->prof_bytes;
        nlaunch[p] = h->prof_n;
        if (2 * nlaunch[p] > (int)h->prof_ev.size()) { rc = fail(h, IBPM_ERR_INVALID, "too many launches"); break; }
    }
    // the events of both graphs are the same objects: replay one step at a time
    CK(cudaMemsetAsync(h->counter, 0, sizeof(int), h->st));
    for (int s = 0; s < nsteps && rc == IBPM_OK; ++s) {
        if (flush_l2) CK(cudaMemsetAsync(h->flush_buf, s & 0xff, h->flush_bytes, h->st));
        const int p = h->cur;
        CK(cudaGraphLaunch(pexec[p], h->st));
        h->cur ^= 1;
        CK(cudaStreamSynchronize(h->st));
        for (int i = 0; i < nlaunch[p]; ++i) {
            float ms = 0;
            CK(cudaEventElapsedTime(&ms, h->prof_ev[2 * i], h->prof_ev[2 * i + 1]));
            ms_out[lab[p][i]] += ms;
            bytes_out[lab[p][i]] += byt[p][i];
            calls_out[lab[p][i]] += 1;
        }
    }
    h->nonlin1_valid = false;
    for (int p = 0; p < 2; ++p) if (pexec[p]) cudaGraphExecDestroy(pexec[p]);
    return rc;
}

// ---------------------------------------------------------------------------
// Discrete adjoint: the transpose of the derivative of one step, checkpointed
// recomputation, and the gradient of a time-averaged force objective.
// ---------------------------------------------------------------------------

// Transpose of the level chain of vort2flux! (curl.jl:147-162), finest level
// first: ψ̄ = curl!ᵀ(q̄) + get_bc!ᵀ(edge adjoint of the finer level), Γ̄ += Δ⁻¹ψ̄
// (Δ⁻¹ is symmetric).  q̄ is given on levels [0, qnlev), zero above.
static int solves_T(ibpm_handle* h, const double* qbar, int qnlev, double* Gacc) {
    const Geom& g = h->g;
    const int mg = g.mg;
    const long long bs = g.S * mg;
    const double slab = 16.0 * g.n1 * g.n2;
    for (int lev = 0; lev < mg; ++lev) {
        LAUNCH(K_ADJ, 8.0 * (g.nq + 2.0 * g.n1 * g.n2),
               launch_adj_curlT(g, lev < qnlev ? qbar + (long long)lev * g.nq : nullptr,
                                lev > 0 ? h->bcc + (long long)(lev - 1) * g.nbc : nullptr,
                                lev > 0 ? h->Wadj + (long long)(lev - 1) * g.S : nullptr, h->psib,
                                h->bcc + (long long)lev * g.nbc, h->st));
        SlabMap one = levmap(g, 0, 1, g.S);
        SlabMap m = levmap(g, lev, 1, bs);
        XPassArgs a{};
        a.in = h->psib; a.out = h->rhs; a.in_map = one; a.out_map = one;
        a.nslabs = 1; a.line0 = 0; a.line1 = g.n2; a.load = XLOAD_PLAIN; a.emit = XEMIT_STORE;
        LAUNCH(K_DSTX, slab, launch_dst_x(g, h->px, a, h->st));
        LAUNCH(K_DSTY, slab, launch_dst_y(g, h->py, h->px, h->rhs, one, 1, spec(h, SPEC_DELTA), h->st));
        XPassArgs c{};
        c.in = h->rhs; c.out = Gacc; c.in_map = one; c.out_map = m; c.aux = h->Wadj; c.aux_map = m;
        c.nslabs = 1; c.line0 = 0; c.line1 = g.n2; c.load = XLOAD_PLAIN; c.emit = XEMIT_ADD_STORE;
        LAUNCH(K_DSTX, slab * 2.0, launch_dst_x(g, h->px, c, h->st));
    }
    return IBPM_OK;
}

// Transpose of the coarsify chain (curl.jl:141-143): coarsest level first.
static int coarsify_T(ibpm_handle* h, double* Gacc) {
    const Geom& g = h->g;
    const int mg = g.mg;
    for (int lev = mg - 1; lev >= 1; --lev)
        LAUNCH(K_ADJ, 8.0 * 2.25 * g.n1 * g.n2,
               launch_adj_coarsifyT(g, Gacc, g.S, lev, lev + 1 <= mg - 1 ? lev + 1 : -1, h->st));
    if (mg >= 2) LAUNCH(K_ADJ, 2.0 * g.n1 * g.n2, launch_zero_centre(g, Gacc + g.S, h->st));
    return IBPM_OK;
}

// Adjoint of one step, from (Γ̄, q̄, N̄[par]) of the next state to those of
// this one (N̄ into N̄[par^1]), with this step's forward (Γ_n, q_n) in tape
// slot (*adj_n mod k) and objective weight stepw[*adj_n].
static int enqueue_adjoint_step(ibpm_handle* h, int par) {
    const Geom& g = h->g;
    const int mg = g.mg;
    const long long bs = g.S * mg;
    int rc;
    // project_circ! and the final vort2flux!: Γ_{n+1} = coarsify(Γ'), q_{n+1} = curl ψ(Γ_{n+1})
    CK(cudaMemcpyAsync(h->Gt, h->Gb, sizeof(double) * bs, cudaMemcpyDeviceToDevice, h->st));
    if ((rc = solves_T(h, h->qb, mg, h->Gt))) return rc;
    if ((rc = coarsify_T(h, h->Gt))) return rc;
    // Γ' = Γs − e₁ A⁻¹₁ C'E' F̃b:  F̄t = ∂J/∂F̃b − E rot!ᵀ(A⁻¹₁ Γ̄'₁)
    SlabMap l0 = levmap(g, 0, 1, bs);
    if ((rc = poisson(h, h->Gt, l0, h->rhs, l0, h->rb, l0, 1, SPEC_AINV, XEMIT_STORE))) return rc;
    LAUNCH(K_ADJ, 16.0 * 169 * h->nf,
           launch_adj_E_rotT(g, h->body, h->rb, h->adj_wx, h->adj_wy, h->stepw, h->adj_n, h->Ft, h->st));
    // F̃b = B⁻¹ E(qs + q0)
    LAUNCH(K_ADJ, 8.0 * h->nf * (h->nf + 2.0), launch_gemv_t(h->Binv, h->Ft, h->Fbar, h->nf, h->st));
    LAUNCH(K_ADJ, 8.0 * 4 * 169 * h->nf,
           launch_adj_Et(g, h->body, h->Fbar, h->qsb, h->q0part + (long long)mg * adj_nlq_blocks(g) * 2, h->st));
    // the trial vort2flux!: Γs ← coarsify(Γs), qs = curl ψs on level 1
    if ((rc = solves_T(h, h->qsb, 1, h->Gt))) return rc;
    if ((rc = coarsify_T(h, h->Gt))) return rc;
    // get_trial_state!: r̄ = A⁻¹ Γ̄s (every level), then the products and stencils
    SlabMap all = levmap(g, 0, mg, bs);
    if ((rc = poisson(h, h->Gt, all, h->rhs, all, h->rb, all, mg, SPEC_AINV, XEMIT_STORE))) return rc;
    AdjTrialArgs ta{};
    ta.rb = h->rb; ta.Nb_in = h->Nb[par]; ta.Nb_out = h->Nb[par ^ 1];
    ta.tapeG = h->tapeG; ta.tapeq = h->tapeq; ta.tape_gstride = bs; ta.tape_qstride = (long long)g.nq * mg;
    ta.adj_n = h->adj_n; ta.k = h->adj_k;
    ta.Gb = h->Gb; ta.qb = h->qb; ta.bcv = h->bcv; ta.q0part = h->q0part;
    const RhsArgs ra = rhs_args(h, 0);
    for (int l = 0; l < mg; ++l) {
        ta.q0x[l] = h->q0x[l]; ta.q0y[l] = h->q0y[l];
        ta.c_lap[l] = ra.c_lap[l]; ta.fac_bc[l] = ra.fac_bc[l]; ta.nl_scale[l] = ra.nl_scale[l];
    }
    ta.b1dt = ra.b1dt; ta.b2dt = ra.b2dt; ta.mg = mg;
    if (h->adj_xb) {
        // ∂J/∂xb of this step: F̄ · ∂E[q_{n+1,1} + q0] − F̃_n · ∂E[C r̄₁]
        AdjXbArgs xa{};
        xa.wd = h->wd; xa.Fbar = h->Fbar; xa.tapeFb = h->tapeFb; xa.tapeq1 = h->tapeq1;
        xa.adj_n = h->adj_n; xa.k = h->adj_k; xa.q0x = h->q0x[0]; xa.q0y = h->q0y[0];
        xa.rb1 = h->rb; xa.gxb = h->gxb;
        LAUNCH(K_ADJ, 8.0 * (4.0 * 169 * h->nf + 2.0 * h->nf), launch_adj_xb(g, h->body, xa, h->st));
    }
    LAUNCH(K_ADJ, 8.0 * (10.0 * g.n1 * g.n2 + 3.0 * g.nq) * mg, launch_adj_trial(g, ta, h->st));
    LAUNCH(K_ADJ, 8.0, launch_adj_tick(h->adj_n, h->st));
    return IBPM_OK;
}

// Buffers of the position gradient for segments of k steps (the adjoint graphs
// hold their pointers: reallocation drops them).
static int xb_alloc(ibpm_handle* h, int k) {
    if (!h->wd) {
        int rc = dalloc(h, &h->wd, (size_t)h->nf * 338);
        if (rc) return rc;
        CK(launch_dweights(h->h, h->offx, h->offy, h->body, h->wd, h->st));
    }
    if (!h->gxb) {
        int rc = dalloc(h, &h->gxb, h->nf);
        if (rc) return rc;
    }
    if (h->xb_k < k) {
        for (int p = 0; p < 2; ++p) if (h->gadj[p]) { cudaGraphExecDestroy(h->gadj[p]); h->gadj[p] = nullptr; }
        if (h->tapeFb) cudaFree(h->tapeFb);
        if (h->tapeq1) cudaFree(h->tapeq1);
        h->tapeFb = h->tapeq1 = nullptr;
        h->xb_k = 0;
        int rc;
        if ((rc = dalloc(h, &h->tapeFb, (size_t)k * h->nf)) || (rc = dalloc(h, &h->tapeq1, (size_t)k * h->g.nq)))
            return rc;
        h->xb_k = k;
    }
    return IBPM_OK;
}

static int adj_alloc(ibpm_handle* h, int k, int ncp, int nsteps) {
    const Geom& g = h->g;
    const long long bs = g.S * g.mg, qs = (long long)g.nq * g.mg;
    const long long ckd = 3 * bs + qs + (h->Pp ? g.S : 0);
    if (h->Gb && k == h->adj_k && ncp <= h->adj_ncp && nsteps <= h->adj_nsteps) return IBPM_OK;
    for (int p = 0; p < 2; ++p) if (h->gadj[p]) { cudaGraphExecDestroy(h->gadj[p]); h->gadj[p] = nullptr; }
    double** bufs[] = {&h->tapeG, &h->tapeq, &h->ck, &h->Gb, &h->qb, &h->Nb[0], &h->Nb[1], &h->Gt, &h->psib,
                       &h->Wadj, &h->rb, &h->qsb, &h->Ft, &h->Fbar, &h->bcc, &h->bcv, &h->q0part, &h->stepw};
    for (double** b : bufs) if (*b) { cudaFree(*b); *b = nullptr; }
    if (h->adj_n) { cudaFree(h->adj_n); h->adj_n = nullptr; }
    int rc;
    const long long nq0 = (long long)g.mg * adj_nlq_blocks(g) * 2 + 2;
    if ((rc = dalloc(h, &h->tapeG, (size_t)k * bs)) || (rc = dalloc(h, &h->tapeq, (size_t)k * qs)) ||
        (rc = dalloc(h, &h->ck, (size_t)(ncp + 1) * ckd)) || (rc = dalloc(h, &h->Gb, bs)) ||
        (rc = dalloc(h, &h->qb, qs)) || (rc = dalloc(h, &h->Nb[0], bs)) || (rc = dalloc(h, &h->Nb[1], bs)) ||
        (rc = dalloc(h, &h->Gt, bs)) || (rc = dalloc(h, &h->psib, g.S)) || (rc = dalloc(h, &h->Wadj, bs)) ||
        (rc = dalloc(h, &h->rb, bs)) || (rc = dalloc(h, &h->qsb, g.nq)) || (rc = dalloc(h, &h->Ft, h->nf)) ||
        (rc = dalloc(h, &h->Fbar, h->nf)) || (rc = dalloc(h, &h->bcc, (size_t)g.mg * g.nbc)) ||
        (rc = dalloc(h, &h->bcv, (size_t)g.mg * g.nbc)) || (rc = dalloc(h, &h->q0part, nq0)) ||
        (rc = dalloc(h, &h->stepw, nsteps)) || (rc = dalloc(h, &h->adj_n, 1)))
        return rc;
    // slab pitch padding, the untouched flux rows of q̄s and unused edge
    // entries must read as zero
    for (double* p : {h->psib, h->Wadj, h->rb, h->Gt, h->Gb, h->Nb[0], h->Nb[1]})
        CK(cudaMemsetAsync(p, 0, sizeof(double) * (p == h->psib ? g.S : bs), h->st));
    CK(cudaMemsetAsync(h->qsb, 0, sizeof(double) * g.nq, h->st));
    CK(cudaMemsetAsync(h->bcv, 0, sizeof(double) * g.mg * g.nbc, h->st));
    h->adj_k = k; h->adj_ncp = ncp; h->adj_nsteps = nsteps; h->ck_doubles = ckd;
    h->ck_cur.assign(ncp + 1, 0);
    h->ck_cold.assign(ncp + 1, 0);
    return IBPM_OK;
}

// Checkpoint slot c <-> the state that a step reads: Γ, q, N_{n-1} of the
// current parity, ψ and the refined mode's projection guess.
static int ck_copy(ibpm_handle* h, int c, bool save) {
    const Geom& g = h->g;
    const long long bs = g.S * g.mg, qs = (long long)g.nq * g.mg;
    double* base = h->ck + (long long)c * h->ck_doubles;
    if (!save) { h->cur = h->ck_cur[c]; h->cold = h->ck_cold[c]; }
    struct { double* dev; long long n; } f[5] = {{h->G[h->cur], bs}, {h->q, qs}, {h->Nl[h->cur], bs}, {h->psi, bs},
                                                 {h->Pp, h->Pp ? g.S : 0}};
    long long off = 0;
    for (auto& x : f) {
        if (!x.n) continue;
        if (save) CK(cudaMemcpyAsync(base + off, x.dev, sizeof(double) * x.n, cudaMemcpyDeviceToDevice, h->st));
        else CK(cudaMemcpyAsync(x.dev, base + off, sizeof(double) * x.n, cudaMemcpyDeviceToDevice, h->st));
        off += x.n;
    }
    if (save) { h->ck_cur[c] = h->cur; h->ck_cold[c] = h->cold; }
    return IBPM_OK;
}

extern "C" int ibpm_adjoint_run(ibpm_handle* h, int32_t nsteps, int32_t k_checkpoint, const ibpm_objective* obj,
                                double* J, double* grad_Gamma0, double* grad_q0, double* grad_omega0,
                                double* grad_alpha, double* grad_xb) {
    if (!h || !obj || nsteps < 1 || k_checkpoint < 1) return IBPM_ERR_INVALID;
    if (obj->window < 1 || obj->window > nsteps) return fail(h, IBPM_ERR_INVALID, "objective window must be in 1..nsteps");
    if (h->lin) return fail(h, IBPM_ERR_UNSUPPORTED, "the adjoint is of the nonlinear step, not of a linearised problem");
    if (h->moving || h->bodies_moving)
        return fail(h, IBPM_ERR_UNSUPPORTED, "the adjoint is of the static-body step, not of moving bodies or grids");
    CK(cudaSetDevice(h->device));
    const Geom& g = h->g;
    const int mg = g.mg;
    const long long bs = g.S * mg, qs = (long long)g.nq * mg;
    const int k = std::min(k_checkpoint, nsteps);
    const int ncp = (nsteps + k - 1) / k;
    int rc = ensure_graphs(h, std::max(std::max(1024, h->hist_cap), k));
    if (rc) return rc;
    if ((rc = adj_alloc(h, k, ncp, nsteps))) return rc;
    h->adj_xb = grad_xb != nullptr;
    if (h->adj_xb && (rc = xb_alloc(h, k))) return rc;
    if (h->gadj_xb != h->adj_xb)  // the captured adjoint step must match the request
        for (int p = 0; p < 2; ++p) if (h->gadj[p]) { cudaGraphExecDestroy(h->gadj[p]); h->gadj[p] = nullptr; }
    h->adj_wx = obj->w_cd * 2.0 * h->h / h->dt;  // CD_j = 2 (h/dt) Σ F̃x (timestepping.jl:330-354)
    h->adj_wy = obj->w_cl * 2.0 * h->h / h->dt;
    std::vector<double> w(nsteps, 0.0);
    for (int n = nsteps - obj->window; n < nsteps; ++n) w[n] = 1.0 / obj->window;
    CK(cudaMemcpyAsync(h->stepw, w.data(), sizeof(double) * nsteps, cudaMemcpyHostToDevice, h->st));
    for (int p = 0; p < 2; ++p)
        if (!h->gadj[p]) {
            cudaGraph_t graph;
            CK(cudaStreamBeginCapture(h->st, cudaStreamCaptureModeThreadLocal));
            rc = enqueue_adjoint_step(h, p);
            cudaError_t e = cudaStreamEndCapture(h->st, &graph);
            if (rc) return rc;
            if (e != cudaSuccess) return fail(h, IBPM_ERR_CUDA, std::string("adjoint capture: ") + cudaGetErrorString(e));
            e = cudaGraphInstantiate(&h->gadj[p], graph, 0);
            cudaGraphDestroy(graph);
            if (e != cudaSuccess) return fail(h, IBPM_ERR_CUDA, std::string("adjoint instantiate: ") + cudaGetErrorString(e));
            h->gadj_xb = h->adj_xb;
        }
    // ---- forward pass with a checkpoint every k steps; J from CD/CL
    CK(cudaMemsetAsync(h->status, 0, sizeof(int), h->st));
    double Jv = 0.0;
    std::vector<double> hb;
    int done = 0;
    while (done < nsteps) {
        const int n = std::min(h->hist_cap, nsteps - done);
        CK(cudaMemsetAsync(h->counter, 0, sizeof(int), h->st));
        for (int s = 0; s < n; ++s) {
            if ((done + s) % k == 0 && (rc = ck_copy(h, (done + s) / k, true))) return rc;
            CK(launch_step(h));
        }
        hb.resize((size_t)n * 2 * h->nbodies);
        CK(cudaMemcpyAsync(hb.data(), h->hist, sizeof(double) * hb.size(), cudaMemcpyDeviceToHost, h->st));
        CK(cudaStreamSynchronize(h->st));
        for (int s = 0; s < n; ++s)
            for (int j = 0; j < h->nbodies; ++j)
                Jv += w[done + s] * (obj->w_cd * hb[((size_t)s * 2 + 0) * h->nbodies + j] +
                                     obj->w_cl * hb[((size_t)s * 2 + 1) * h->nbodies + j]);
        done += n;
    }
    if ((rc = ck_copy(h, ncp, true))) return rc;  // the final state, restored at the end
    // ---- reverse sweep: recompute each segment into the tape, then adjoint steps
    for (double* p : {h->Gb, h->Nb[0], h->Nb[1]}) CK(cudaMemsetAsync(p, 0, sizeof(double) * bs, h->st));
    CK(cudaMemsetAsync(h->qb, 0, sizeof(double) * qs, h->st));
    const long long nq0 = (long long)mg * adj_nlq_blocks(g) * 2 + 2;
    CK(cudaMemsetAsync(h->q0part, 0, sizeof(double) * nq0, h->st));
    if (h->adj_xb) CK(cudaMemsetAsync(h->gxb, 0, sizeof(double) * h->nf, h->st));
    const int last = nsteps - 1;
    CK(cudaMemcpyAsync(h->adj_n, &last, sizeof(int), cudaMemcpyHostToDevice, h->st));
    int par = 0;
    for (int c = ncp - 1; c >= 0; --c) {
        const int s0 = c * k, s1 = std::min(s0 + k, nsteps);
        if ((rc = ck_copy(h, c, false))) return rc;
        CK(cudaMemsetAsync(h->counter, 0, sizeof(int), h->st));
        for (int n = s0; n < s1; ++n) {
            const int slot = n % k;
            CK(cudaMemcpyAsync(h->tapeG + slot * bs, h->G[h->cur], sizeof(double) * bs, cudaMemcpyDeviceToDevice,
                               h->st));
            CK(cudaMemcpyAsync(h->tapeq + slot * qs, h->q, sizeof(double) * qs, cudaMemcpyDeviceToDevice, h->st));
            CK(launch_step(h));
            if (h->adj_xb) {  // what the position gradient reads: F̃b and the level-1 q the step produced
                CK(cudaMemcpyAsync(h->tapeFb + (long long)slot * h->nf, h->Fb, sizeof(double) * h->nf,
                                   cudaMemcpyDeviceToDevice, h->st));
                CK(cudaMemcpyAsync(h->tapeq1 + (long long)slot * g.nq, h->q, sizeof(double) * g.nq,
                                   cudaMemcpyDeviceToDevice, h->st));
            }
        }
        for (int n = s1 - 1; n >= s0; --n) {
            CK(cudaGraphLaunch(h->gadj[par], h->st));
            par ^= 1;
        }
    }
    // ---- gradients with respect to the initial state
    CK(cudaStreamSynchronize(h->st));
    if (J) *J = Jv;
    auto slabs_out = [&](double* dst, const double* src) {
        const size_t wbytes = sizeof(double) * g.n1, rows = (size_t)g.n2 * mg;
        return cudaMemcpy2DAsync(dst, wbytes, src, sizeof(double) * g.P, wbytes, rows, cudaMemcpyDeviceToHost, h->st);
    };
    if (grad_Gamma0) CK(slabs_out(grad_Gamma0, h->Gb));
    if (grad_q0) CK(cudaMemcpyAsync(grad_q0, h->qb, sizeof(double) * qs, cudaMemcpyDeviceToHost, h->st));
    if (grad_omega0) {
        // Γ₀ = coarsify([h²ω, 0, …]), q₀ = curl ψ(Γ₀): ω̄ = h² (coarsify!ᵀ(Γ̄₀ + solves!ᵀ(q̄₀)))₁
        CK(cudaMemcpyAsync(h->Gt, h->Gb, sizeof(double) * bs, cudaMemcpyDeviceToDevice, h->st));
        if ((rc = solves_T(h, h->qb, mg, h->Gt)) || (rc = coarsify_T(h, h->Gt))) return rc;
        std::vector<double> G1((size_t)g.n1 * g.n2);
        const size_t wbytes = sizeof(double) * g.n1;
        CK(cudaMemcpy2DAsync(G1.data(), wbytes, h->Gt, sizeof(double) * g.P, wbytes, g.n2, cudaMemcpyDeviceToHost,
                             h->st));
        CK(cudaStreamSynchronize(h->st));
        for (size_t i = 0; i < G1.size(); ++i) grad_omega0[i] = h->h * h->h * G1[i];
    }
    if (grad_alpha) {
        // q0x = (Ux cos α − Uy sin α) hc, q0y = (Ux sin α + Uy cos α) hc (timestepping.jl:252-270)
        std::vector<double> part(nq0);
        CK(cudaMemcpyAsync(part.data(), h->q0part, sizeof(double) * nq0, cudaMemcpyDeviceToHost, h->st));
        CK(cudaStreamSynchronize(h->st));
        const int nb = adj_nlq_blocks(g);
        double d = 0.0;
        for (int l = 0; l < mg; ++l) {
            double sx = 0.0, sy = 0.0;
            for (int b = 0; b < nb; ++b) { sx += part[2 * ((size_t)l * nb + b)]; sy += part[2 * ((size_t)l * nb + b) + 1]; }
            if (l == 0) { sx += part[nq0 - 2]; sy += part[nq0 - 1]; }
            const double hc = h->h * std::ldexp(1.0, l), a = h->incl;
            d += sx * (-h->Ux * std::sin(a) - h->Uy * std::cos(a)) * hc;
            d += sy * (h->Ux * std::cos(a) - h->Uy * std::sin(a)) * hc;
        }
        *grad_alpha = d;
    }
    if (grad_xb) CK(cudaMemcpyAsync(grad_xb, h->gxb, sizeof(double) * h->nf, cudaMemcpyDeviceToHost, h->st));
    if ((rc = ck_copy(h, ncp, false))) return rc;  // leave the handle at the final state
    CK(cudaStreamSynchronize(h->st));
    int hstatus = 0;
    CK(cudaMemcpy(&hstatus, h->status, sizeof(int), cudaMemcpyDeviceToHost));
    if (hstatus) return fail(h, IBPM_ERR_NONFINITE, "CD/CL became non-finite");
    return IBPM_OK;
}

// Time the adjoint step alone: graph replays of the adjoint of one step
// (tape slot 0 repeatedly), CUDA events around each.
extern "C" int ibpm_adjoint_bench(ibpm_handle* h, int32_t nsteps, int32_t flush_l2, double* step_ms) {
    if (!h || nsteps < 1 || !step_ms) return IBPM_ERR_INVALID;
    if (!h->gadj[0] || !h->gadj[1]) return fail(h, IBPM_ERR_INVALID, "no adjoint captured: run ibpm_adjoint_run first");
    CK(cudaSetDevice(h->device));
    if (flush_l2 && !h->flush_buf) {
        h->flush_bytes = (size_t)512 << 20;
        int rc = dalloc(h, (char**)&h->flush_buf, h->flush_bytes);
        if (rc) return rc;
    }
    const int zero = 0;
    std::vector<cudaEvent_t> ev(2 * nsteps);
    for (auto& e : ev) CK(cudaEventCreate(&e));
    for (int s = 0; s < nsteps; ++s) {
        CK(cudaMemcpyAsync(h->adj_n, &zero, sizeof(int), cudaMemcpyHostToDevice, h->st));
        if (flush_l2) CK(cudaMemsetAsync(h->flush_buf, s & 0xff, h->flush_bytes, h->st));
        CK(cudaEventRecord(ev[2 * s], h->st));
        CK(cudaGraphLaunch(h->gadj[s & 1], h->st));
        CK(cudaEventRecord(ev[2 * s + 1], h->st));
    }
    CK(cudaStreamSynchronize(h->st));
    for (int s = 0; s < nsteps; ++s) {
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, ev[2 * s], ev[2 * s + 1]));
        step_ms[s] = ms;
    }
    for (auto& e : ev) cudaEventDestroy(e);
    return IBPM_OK;
}

// ---------------------------------------------------------------------------
// Batches of independent simulations.  Each member is an ordinary handle;
// one step of the batch is one graph launch whose branches are the steps of
// its units, spread over `lanes` concurrent streams (units of one lane run one
// after another).  A unit is one member, or (grouped) a group of members of
// one grid, precision, level chain and plan, whose step fields sit in shared
// arenas: the group's transforms and stencils are launches over the slabs of
// all its members, its body operators one short branch per member.  Small
// grids leave most of the GPU idle when run alone; side by side and in shared
// launches they fill it.  Lanes, plan, chain and grouping are picked by
// timing.
// ---------------------------------------------------------------------------
struct BatchGroup {
    std::vector<ibpm_handle*> mem;             // lead first
    std::vector<std::pair<char*, size_t>> arenas;  // step fields, member after member (base, bytes)
    double* den = nullptr;                     // [n][9] spectral factors (SpecParams::mden)
    double* cA = nullptr;                      // [n]
    RhsArgs* rhs[2] = {nullptr, nullptr};      // [n] per parity
    std::vector<cudaStream_t> br;              // branch streams of the body operators
    std::vector<cudaEvent_t> ev;               // fork + one join event per member
};

struct ibpm_batch {
    std::vector<BatchGroup> groups;
    bool grouped = true;                       // groups step by shared launches
    int device = 0;
    std::vector<ibpm_handle*> m;
    cudaStream_t st = nullptr;                 // the batch stream (fork/join point)
    std::vector<cudaStream_t> lane_st;
    std::vector<cudaEvent_t> ev;               // fork + one join event per lane
    int lanes = 0;
    int plan = IBPM_PLAN_LATENCY;              // transform plan of the members' single-slab launches
    int chain = IBPM_CHAIN_BOUNDARY_TRANSFER;  // the members' level chain
    int cur = 0;                               // parity shared by the members
    int cold = kColdSteps;
    cudaGraphExec_t g[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};  // [cold][parity]
    int hist_cap = 0;
    std::vector<double> cd, cl;                // [member][step][body] of the last advance
    std::vector<int> off;                      // member offsets into cd/cl
    int last_steps = 0;
    std::string err;
};

static int bfail(ibpm_batch* b, int code, const std::string& msg) {
    b->err = msg;
    return code;
}

#define BCK(call)                                                                          \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess) return bfail(b, IBPM_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

// Zero the state of a handle, as after create.
static int reset_state(ibpm_handle* h) {
    const Geom& g = h->g;
    const size_t slabs = (size_t)g.S * g.mg;
    for (double* p : {h->G[0], h->G[1], h->Nl[0], h->Nl[1], h->psi, h->nonlin1_shadow})
        CK(cudaMemsetAsync(p, 0, sizeof(double) * slabs, h->st));
    CK(cudaMemsetAsync(h->q, 0, sizeof(double) * g.nq * g.mg, h->st));
    CK(cudaMemsetAsync(h->Fb, 0, sizeof(double) * h->nf, h->st));
    if (h->Pp) CK(cudaMemsetAsync(h->Pp, 0, sizeof(double) * g.S, h->st));
    CK(cudaStreamSynchronize(h->st));
    h->cur = 0;
    h->cold = kColdSteps;
    h->nonlin1_valid = false;
    return IBPM_OK;
}

static void batch_free_graphs(ibpm_batch* b) {
    for (auto& row : b->g)
        for (auto& x : row)
            if (x) { cudaGraphExecDestroy(x); x = nullptr; }
}

// The step fields of a group's members moved into arenas, member after member
// with the strides the shared launches assume: mg slabs for every slab field
// (Gsrc and Pp included, though they use one), nq·mg for q and qs, and the
// boundary-transfer vectors at their per-simulation sizes.  The content is
// kept; each member then points into the arenas.
template <class T, class F>
static cudaError_t rehome(BatchGroup& gr, F field, size_t per, size_t have, cudaStream_t st) {
    if (!field(gr.mem[0])) return cudaSuccess;   // a field this precision does not use
    const size_t n = gr.mem.size();
    T* a = nullptr;
    cudaError_t e = cudaMalloc((void**)&a, sizeof(T) * per * n);
    if (e != cudaSuccess) return e;
    gr.arenas.push_back({reinterpret_cast<char*>(a), sizeof(T) * per * n});
    if ((e = cudaMemsetAsync(a, 0, sizeof(T) * per * n, st)) != cudaSuccess) return e;
    for (size_t i = 0; i < n; ++i)
        if ((e = cudaMemcpyAsync(a + i * per, field(gr.mem[i]), sizeof(T) * have, cudaMemcpyDeviceToDevice, st)) !=
            cudaSuccess)
            return e;
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return e;
    for (size_t i = 0; i < n; ++i) {
        cudaFree(field(gr.mem[i]));
        field(gr.mem[i]) = a + i * per;
    }
    return cudaSuccess;
}

// The fields of a handle that point into the group's arenas, set to nullptr
// before the arenas are freed.  A field the group did not move (an arena
// allocation failed part way) stays with the handle, which releases it.
static void forget_arena_fields(ibpm_handle* h, const BatchGroup& gr) {
    auto drop = [&](auto*& p) {
        const char* c = reinterpret_cast<const char*>(p);
        for (const auto& a : gr.arenas)
            if (c && c >= a.first && c < a.first + a.second) { p = nullptr; return; }
    };
    drop(h->G[0]); drop(h->G[1]); drop(h->Nl[0]); drop(h->Nl[1]);
    drop(h->psi); drop(h->q); drop(h->qs); drop(h->rhs); drop(h->Gsrc); drop(h->Pp);
    drop(h->T32);
    drop(h->btY); drop(h->btS); drop(h->btE); drop(h->btP);
    drop(h->btY32);
}

static int batch_make_group(ibpm_batch* b, const std::vector<ibpm_handle*>& mem) {
    b->groups.emplace_back();
    BatchGroup& gr = b->groups.back();
    gr.mem = mem;
    ibpm_handle* h0 = mem[0];
    const Geom& g = h0->g;
    const int mg = g.mg, n = (int)mem.size();
    const size_t slabs = (size_t)g.S * mg, nq = (size_t)g.nq * mg;
    cudaStream_t st = b->st;
    cudaError_t e = cudaSuccess;
    using D = double;
    auto rd = [&](auto field, size_t per, size_t have) {
        if (e == cudaSuccess) e = rehome<D>(gr, field, per, have, st);
    };
    auto rf = [&](auto field, size_t per, size_t have) {
        if (e == cudaSuccess) e = rehome<float>(gr, field, per, have, st);
    };
    rd([](ibpm_handle* h) -> double*& { return h->G[0]; }, slabs, slabs);
    rd([](ibpm_handle* h) -> double*& { return h->G[1]; }, slabs, slabs);
    rd([](ibpm_handle* h) -> double*& { return h->Nl[0]; }, slabs, slabs);
    rd([](ibpm_handle* h) -> double*& { return h->Nl[1]; }, slabs, slabs);
    rd([](ibpm_handle* h) -> double*& { return h->psi; }, slabs, slabs);
    rd([](ibpm_handle* h) -> double*& { return h->rhs; }, slabs, slabs);
    rd([](ibpm_handle* h) -> double*& { return h->Gsrc; }, slabs, (size_t)g.S);
    rd([](ibpm_handle* h) -> double*& { return h->Pp; }, slabs, (size_t)g.S);
    rd([](ibpm_handle* h) -> double*& { return h->q; }, nq, nq);
    rd([](ibpm_handle* h) -> double*& { return h->qs; }, nq, nq);
    rf([](ibpm_handle* h) -> float*& { return h->T32; }, slabs, slabs);
    rd([](ibpm_handle* h) -> double*& { return h->btY; }, slabs, slabs);
    rf([](ibpm_handle* h) -> float*& { return h->btY32; }, slabs, slabs);
    const size_t nsmp = (size_t)bt_sample_len(g) * mg, ne = (size_t)bt_edge_pitch(g) * mg;
    const size_t np = (size_t)(mg - 1) * h0->bt_kp;
    rd([](ibpm_handle* h) -> double*& { return h->btS; }, nsmp, nsmp);
    rd([](ibpm_handle* h) -> double*& { return h->btE; }, ne, ne);
    if (np) rd([](ibpm_handle* h) -> double*& { return h->btP; }, np, np);
    for (auto* h : mem) { h->arena = true; h->graphs_ready = false; }
    if (e != cudaSuccess) return bfail(b, IBPM_ERR_NOMEM, std::string("batch group arenas: ") + cudaGetErrorString(e));
    BCK(cudaMalloc((void**)&gr.den, sizeof(double) * 9 * n));
    BCK(cudaMalloc((void**)&gr.cA, sizeof(double) * n));
    for (int p = 0; p < 2; ++p) BCK(cudaMalloc((void**)&gr.rhs[p], sizeof(RhsArgs) * n));
    gr.br.resize(n);
    gr.ev.resize(n + 1);
    for (auto& x : gr.br) BCK(cudaStreamCreateWithFlags(&x, cudaStreamNonBlocking));
    for (auto& x : gr.ev) BCK(cudaEventCreateWithFlags(&x, cudaEventDisableTiming));
    return IBPM_OK;
}

// Members of one grid (nx, ny, mg), precision, sweep count and boundary-
// transfer rank, with fixed bodies on a fixed grid, form a group (two or more).
static int batch_make_groups(ibpm_batch* b) {
    std::map<std::vector<int>, std::vector<ibpm_handle*>> keys;
    for (auto* h : b->m) {
        if (h->moving || h->bodies_moving || h->lin) continue;
        keys[{h->g.nx, h->g.ny, h->g.mg, h->prec, h->sweeps, h->btW ? h->bt_kp : -1}].push_back(h);
    }
    for (auto& kv : keys)
        if (kv.second.size() >= 2) {
            int rc = batch_make_group(b, kv.second);
            if (rc) return rc;
        }
    return IBPM_OK;
}

static void batch_free_groups(ibpm_batch* b) {
    for (auto& gr : b->groups) {
        for (auto* h : gr.mem) forget_arena_fields(h, gr);
        for (const auto& a : gr.arenas) cudaFree(a.first);
        if (gr.den) cudaFree(gr.den);
        if (gr.cA) cudaFree(gr.cA);
        for (auto* r : gr.rhs) if (r) cudaFree(r);
        for (auto x : gr.br) if (x) cudaStreamDestroy(x);
        for (auto x : gr.ev) if (x) cudaEventDestroy(x);
    }
    b->groups.clear();
}

// A group steps by shared launches when its members agree on everything the
// launches fix (level chain, plans); otherwise its members step one by one.
static bool group_shared(const BatchGroup& gr) {
    const ibpm_handle* h0 = gr.mem[0];
    for (auto* h : gr.mem)
        if (h->bt != h0->bt || h->px.plan1 != h0->px.plan1 || h->px.planN != h0->px.planN ||
            h->py.plan1 != h0->py.plan1 || h->py.planN != h0->py.planN || h->lin || h->moving || h->bodies_moving)
            return false;
    return true;
}

// The per-member tables of a group's shared launches, from the members'
// present problem data (uploaded before each capture).
static int group_tables(ibpm_batch* b, BatchGroup& gr) {
    const int n = (int)gr.mem.size();
    std::vector<double> den(9 * (size_t)n), cA(n);
    std::vector<RhsArgs> ra[2] = {std::vector<RhsArgs>(n), std::vector<RhsArgs>(n)};
    for (int i = 0; i < n; ++i) {
        ibpm_handle* h = gr.mem[i];
        const SpecParams sp = spec(h, SPEC_AINV);
        for (int l = 0; l < 8; ++l) den[9 * i + l] = sp.den[l];
        den[9 * i + 8] = sp.dt;
        cA[i] = c_lap(h, 0);
        for (int p = 0; p < 2; ++p) {
            ra[p][i] = rhs_args(h, p);
            ra[p][i].rhs = h->rhs;
        }
    }
    BCK(cudaMemcpy(gr.den, den.data(), sizeof(double) * den.size(), cudaMemcpyHostToDevice));
    BCK(cudaMemcpy(gr.cA, cA.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
    for (int p = 0; p < 2; ++p)
        BCK(cudaMemcpy(gr.rhs[p], ra[p].data(), sizeof(RhsArgs) * n, cudaMemcpyHostToDevice));
    return IBPM_OK;
}

// The units of a batch step: shared groups (when grouped), then every member
// not in one.  Entries >= 0 are member indices, < 0 group -1 - index.
static std::vector<int> batch_units(ibpm_batch* b) {
    std::vector<int> units;
    std::vector<char> done(b->m.size(), 0);
    if (b->grouped)
        for (size_t k = 0; k < b->groups.size(); ++k)
            if (group_shared(b->groups[k])) {
                units.push_back(-1 - (int)k);
                for (auto* h : b->groups[k].mem)
                    for (size_t i = 0; i < b->m.size(); ++i) if (b->m[i] == h) done[i] = 1;
            }
    for (size_t i = 0; i < b->m.size(); ++i) if (!done[i]) units.push_back((int)i);
    return units;
}

// Enqueue one unit's step on stream `st` (a member, or a group by its lead).
static int batch_enqueue_unit(ibpm_batch* b, int u, cudaStream_t st, int p, bool cold) {
    if (u >= 0) {
        ibpm_handle* h = b->m[u];
        if (h->moving || h->bodies_moving) return bfail(b, IBPM_ERR_UNSUPPORTED, "member " + std::to_string(u) + " moves (not batched)");
        cudaStream_t own = h->st;
        h->st = st;                            // the member's launches join the lane
        const int rc = enqueue_step(h, p, cold);
        h->st = own;
        if (rc) b->err = "member " + std::to_string(u) + ": " + h->err;
        return rc;
    }
    BatchGroup& gr = b->groups[-1 - u];
    ibpm_handle* h = gr.mem[0];
    cudaStream_t own = h->st;
    h->st = st;
    h->gsim = (int)gr.mem.size(); h->gmem = gr.mem.data();
    h->px.sims = h->py.sims = h->gsim;
    h->g_den = gr.den; h->g_cA = gr.cA; h->g_rhs[0] = gr.rhs[0]; h->g_rhs[1] = gr.rhs[1];
    h->g_br = gr.br.data(); h->g_ev = gr.ev.data();
    const int rc = enqueue_step(h, p, cold);
    h->st = own;
    h->gsim = 1; h->gmem = nullptr; h->g_den = nullptr; h->g_cA = nullptr;
    h->px.sims = h->py.sims = 0;
    h->g_rhs[0] = h->g_rhs[1] = nullptr; h->g_br = nullptr; h->g_ev = nullptr;
    if (rc) b->err = "group of " + std::to_string(gr.mem.size()) + " members: " + h->err;
    return rc;
}

// Capture the batch step of parity p (cold: the refined members' first steps).
static int batch_capture(ibpm_batch* b, int lanes, int p, bool cold, cudaGraphExec_t* out) {
    cudaGraph_t graph;
    BCK(cudaStreamBeginCapture(b->st, cudaStreamCaptureModeThreadLocal));
    cudaError_t e = cudaEventRecord(b->ev[0], b->st);
    int rc = IBPM_OK;
    const std::vector<int> units = batch_units(b);
    for (int l = 0; l < lanes && e == cudaSuccess && rc == IBPM_OK; ++l) {
        e = cudaStreamWaitEvent(b->lane_st[l], b->ev[0], 0);
        for (size_t i = l; i < units.size() && e == cudaSuccess && rc == IBPM_OK; i += lanes)
            rc = batch_enqueue_unit(b, units[i], b->lane_st[l], p, cold);
        if (e == cudaSuccess) e = cudaEventRecord(b->ev[1 + l], b->lane_st[l]);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(b->st, b->ev[1 + l], 0);
    }
    cudaError_t ee = cudaStreamEndCapture(b->st, &graph);
    if (rc) return rc;
    if (e != cudaSuccess || ee != cudaSuccess)
        return bfail(b, IBPM_ERR_CUDA, std::string("batch capture: ") + cudaGetErrorString(e != cudaSuccess ? e : ee));
    e = cudaGraphInstantiate(out, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return bfail(b, IBPM_ERR_CUDA, std::string("batch instantiate: ") + cudaGetErrorString(e));
    return IBPM_OK;
}

static int batch_graphs(ibpm_batch* b, int lanes) {
    batch_free_graphs(b);
    for (auto& gr : b->groups) {
        int rc = group_tables(b, gr);
        if (rc) return rc;
    }
    bool any_refined = false;
    for (auto* h : b->m) any_refined |= h->prec == IBPM_PREC_FP32_REFINED;
    for (int c = 0; c < (any_refined ? 2 : 1); ++c)
        for (int p = 0; p < 2; ++p) {
            int rc = batch_capture(b, lanes, p, c == 1, &b->g[c][p]);
            if (rc) return rc;
        }
    b->lanes = lanes;
    return IBPM_OK;
}

static cudaError_t batch_step(ibpm_batch* b) {
    cudaGraphExec_t ge = (b->cold > 0 && b->g[1][b->cur]) ? b->g[1][b->cur] : b->g[0][b->cur];
    if (b->cold > 0) --b->cold;
    const cudaError_t e = cudaGraphLaunch(ge, b->st);
    b->cur ^= 1;
    for (auto* h : b->m) { h->cur = b->cur; h->cold = b->cold; h->nonlin1_valid = false; }
    return e;
}

static void batch_destroy_impl(ibpm_batch* b) {
    if (!b) return;
    if (b->st) cudaStreamSynchronize(b->st);
    batch_free_graphs(b);
    batch_free_groups(b);
    for (auto* h : b->m) { if (h) { cudaStreamSynchronize(h->st); free_handle(h); } }
    for (auto s : b->lane_st) cudaStreamDestroy(s);
    for (auto e : b->ev) cudaEventDestroy(e);
    if (b->st) cudaStreamDestroy(b->st);
    delete b;
}

// Device time of `steps` batch steps with `lanes` lanes (after two untimed).
static int batch_time(ibpm_batch* b, int lanes, int steps, cudaEvent_t e0, cudaEvent_t e1, float* ms) {
    int rc = batch_graphs(b, lanes);
    if (rc) return rc;
    if (steps + 2 > b->hist_cap) return bfail(b, IBPM_ERR_INVALID, "batch tuning: more steps than the force history holds");
    for (auto* h : b->m) BCK(cudaMemsetAsync(h->counter, 0, sizeof(int), b->st));   // the force history restarts
    for (int s = 0; s < 2; ++s)
        if (batch_step(b) != cudaSuccess) return bfail(b, IBPM_ERR_CUDA, "batch tuning step failed");
    cudaEventRecord(e0, b->st);
    for (int s = 0; s < steps; ++s)
        if (batch_step(b) != cudaSuccess) return bfail(b, IBPM_ERR_CUDA, "batch tuning step failed");
    cudaEventRecord(e1, b->st);
    if (cudaEventSynchronize(e1) != cudaSuccess) return bfail(b, IBPM_ERR_CUDA, "batch tuning sync failed");
    cudaEventElapsedTime(ms, e0, e1);
    return IBPM_OK;
}

// Level chain and single-slab plan of some members; false if one of them
// cannot take the chain.
static bool set_members(const std::vector<ibpm_handle*>& mem, int chain, int plan) {
    for (auto* h : mem) {
        if (set_chain(h, chain) != IBPM_OK) return false;
        set_plans(h, plan, h->px.planN);
    }
    return true;
}

// Time `steps` batch steps for each candidate: shared launches or not, the
// members' level chain (sequential or boundary transfer), the transform plan
// of their single-slab launches (latency or throughput) and the lane count
// (powers of two up to the number of units); keep the fastest.  With shared
// launches, each group (largest first) then tries the other chains and plans
// on its own, the batch's other settings fixed, and keeps one that shortens
// the batch step by more than 1%: groups of different grids want different
// ones (the step time is the longest group's chain of launches).  The members
// are reset afterwards.
static int batch_tune(ibpm_batch* b, int steps) {
    struct Cand { int chain, plan, lanes; bool grouped; };
    std::vector<Cand> cand;
    for (bool grp : {true, false}) {
        if (grp && b->groups.empty()) continue;
        b->grouped = grp;
        const int nu = (int)batch_units(b).size();    // the members' chains and plans do not change the units
        for (int ch : {IBPM_CHAIN_SEQUENTIAL, IBPM_CHAIN_BOUNDARY_TRANSFER})
            for (int pl : {IBPM_PLAN_LATENCY, IBPM_PLAN_THROUGHPUT}) {
                for (int l = 1; l < nu; l *= 2) cand.push_back({ch, pl, l, grp});
                cand.push_back({ch, pl, nu, grp});
            }
    }
    double best = 1e300;
    Cand win{IBPM_CHAIN_SEQUENTIAL, IBPM_PLAN_LATENCY, (int)b->m.size(), false};
    cudaEvent_t e0, e1;
    BCK(cudaEventCreate(&e0));
    BCK(cudaEventCreate(&e1));
    int rc = IBPM_OK;
    for (const Cand& c : cand) {
        if (!set_members(b->m, c.chain, c.plan)) continue;   // no boundary-transfer factors for a member
        b->grouped = c.grouped;
        float ms = 0;
        if ((rc = batch_time(b, c.lanes, steps, e0, e1, &ms))) break;
        if (ms < best) { best = ms; win = c; }
    }
    if (rc == IBPM_OK && !set_members(b->m, win.chain, win.plan)) rc = bfail(b, IBPM_ERR_CUDA, "batch tuning: level chain");
    b->grouped = win.grouped;
    if (rc == IBPM_OK && win.grouped) {
        std::vector<int> order(b->groups.size());
        for (size_t k = 0; k < order.size(); ++k) order[k] = (int)k;
        auto cells = [&](int k) {
            const Geom& g = b->groups[k].mem[0]->g;
            return (double)g.nx * g.ny * g.mg * b->groups[k].mem.size();
        };
        std::sort(order.begin(), order.end(), [&](int x, int y) { return cells(x) > cells(y); });
        float base = 0;
        rc = batch_time(b, win.lanes, 2 * steps, e0, e1, &base);
        for (int k : order) {
            if (rc) break;
            const auto& mem = b->groups[k].mem;
            const int ch0 = mem[0]->chain, pl0 = mem[0]->px.plan1;
            int keep_ch = ch0, keep_pl = pl0;
            for (int ch : {IBPM_CHAIN_SEQUENTIAL, IBPM_CHAIN_BOUNDARY_TRANSFER})
                for (int pl : {IBPM_PLAN_LATENCY, IBPM_PLAN_THROUGHPUT}) {
                    if (rc || (ch == ch0 && pl == pl0) || !set_members(mem, ch, pl)) continue;
                    float ms = 0;
                    if ((rc = batch_time(b, win.lanes, 2 * steps, e0, e1, &ms))) break;
                    if (ms < 0.99f * base) { base = ms; keep_ch = ch; keep_pl = pl; }
                }
            if (rc == IBPM_OK && !set_members(mem, keep_ch, keep_pl)) rc = bfail(b, IBPM_ERR_CUDA, "batch tuning: level chain");
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    for (auto* h : b->m) {
        if ((rc = reset_state(h))) return bfail(b, rc, h->err);
        if ((rc = ensure_graphs(h, b->hist_cap))) return bfail(b, rc, h->err);  // the members' own graphs
    }
    b->cur = 0;
    b->cold = 2;
    b->plan = win.plan;
    b->chain = win.chain;
    return batch_graphs(b, win.lanes);
}

extern "C" int ibpm_batch_create(int32_t n, const ibpm_problem_desc* descs, int32_t lanes, ibpm_batch** out) {
    if (!out || !descs || n < 1) { g_create_err = "batch: n >= 1 descriptions and an output pointer are required"; return IBPM_ERR_INVALID; }
    *out = nullptr;
    if (lanes < 0 || lanes > n) { g_create_err = "batch: lanes must be in 0..n (0 = tune)"; return IBPM_ERR_INVALID; }
    ibpm_batch* b = new ibpm_batch();
    b->device = descs[0].device;
    for (int i = 0; i < n; ++i) {
        if (descs[i].device != b->device) {
            g_create_err = "batch: all members must be on one device";
            batch_destroy_impl(b);
            return IBPM_ERR_INVALID;
        }
        ibpm_handle* h = nullptr;
        int rc = ibpm_create(&descs[i], &h);
        if (rc) {
            g_create_err = "batch member " + std::to_string(i) + ": " + g_create_err;
            batch_destroy_impl(b);
            return rc;
        }
        b->m.push_back(h);
    }
    int rc = IBPM_OK;
    auto done = [&](int code) {
        if (code) { g_create_err = b->err; batch_destroy_impl(b); return code; }
        *out = b;
        return IBPM_OK;
    };
    if (cudaSetDevice(b->device) != cudaSuccess || cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking) != cudaSuccess)
        return done(bfail(b, IBPM_ERR_CUDA, "batch stream"));
    b->lane_st.resize(n);
    b->ev.resize(n + 1);
    for (int i = 0; i < n; ++i)
        if (cudaStreamCreateWithFlags(&b->lane_st[i], cudaStreamNonBlocking) != cudaSuccess)
            return done(bfail(b, IBPM_ERR_CUDA, "batch lane stream"));
    for (auto& e : b->ev)
        if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess)
            return done(bfail(b, IBPM_ERR_CUDA, "batch event"));
    for (auto* h : b->m) h->in_batch = true;
    if ((rc = batch_make_groups(b))) return done(rc);
    b->hist_cap = 1024;
    for (auto* h : b->m)
        if ((rc = ensure_graphs(h, b->hist_cap))) return done(bfail(b, rc, h->err));
    b->off.assign(n + 1, 0);
    for (int i = 0; i < n; ++i) b->off[i + 1] = b->off[i] + b->m[i]->nbodies;
    rc = lanes == 0 ? batch_tune(b, 8) : batch_graphs(b, lanes);
    return done(rc);
}

extern "C" int ibpm_batch_destroy(ibpm_batch* b) {
    if (!b) return IBPM_ERR_INVALID;
    cudaSetDevice(b->device);
    batch_destroy_impl(b);
    return IBPM_OK;
}

extern "C" ibpm_handle* ibpm_batch_member(ibpm_batch* b, int32_t i) {
    if (!b || i < 0 || i >= (int)b->m.size()) return nullptr;
    return b->m[i];
}

extern "C" int ibpm_batch_lanes(const ibpm_batch* b) { return b ? b->lanes : IBPM_ERR_INVALID; }

extern "C" int ibpm_batch_plan(const ibpm_batch* b) { return b ? b->plan : IBPM_ERR_INVALID; }

extern "C" int ibpm_batch_set_plan(ibpm_batch* b, int32_t plan) {
    if (!b || (plan != IBPM_PLAN_LATENCY && plan != IBPM_PLAN_THROUGHPUT)) return IBPM_ERR_INVALID;
    BCK(cudaSetDevice(b->device));
    BCK(cudaStreamSynchronize(b->st));
    for (auto* h : b->m) {
        set_plans(h, plan, h->px.planN);
        const int rc = ensure_graphs(h, b->hist_cap);   // the members' own graphs
        if (rc) return bfail(b, rc, h->err);
    }
    b->plan = plan;
    return batch_graphs(b, b->lanes);
}

extern "C" int ibpm_batch_chain(const ibpm_batch* b) { return b ? b->chain : IBPM_ERR_INVALID; }

extern "C" int ibpm_batch_grouped(const ibpm_batch* b) { return b ? (b->grouped ? 1 : 0) : IBPM_ERR_INVALID; }

extern "C" int ibpm_batch_set_grouped(ibpm_batch* b, int32_t on) {
    if (!b || (on != 0 && on != 1)) return IBPM_ERR_INVALID;
    BCK(cudaSetDevice(b->device));
    BCK(cudaStreamSynchronize(b->st));
    b->grouped = on == 1;
    return batch_graphs(b, std::min(b->lanes, (int)batch_units(b).size()));
}

extern "C" int ibpm_batch_set_chain(ibpm_batch* b, int32_t chain) {
    if (!b || (chain != IBPM_CHAIN_SEQUENTIAL && chain != IBPM_CHAIN_BOUNDARY_TRANSFER)) return IBPM_ERR_INVALID;
    BCK(cudaSetDevice(b->device));
    BCK(cudaStreamSynchronize(b->st));
    for (size_t i = 0; i < b->m.size(); ++i) {
        ibpm_handle* h = b->m[i];
        int rc = set_chain(h, chain);
        if (rc == IBPM_OK) rc = ensure_graphs(h, b->hist_cap);   // the members' own graphs
        if (rc) return bfail(b, rc, "member " + std::to_string(i) + ": " + h->err);
    }
    b->chain = chain;
    return batch_graphs(b, b->lanes);
}

extern "C" int ibpm_batch_set_lanes(ibpm_batch* b, int32_t lanes) {
    if (!b || lanes < 1 || lanes > (int)b->m.size()) return IBPM_ERR_INVALID;
    BCK(cudaSetDevice(b->device));
    BCK(cudaStreamSynchronize(b->st));
    return batch_graphs(b, lanes);
}

extern "C" const char* ibpm_batch_last_error(const ibpm_batch* b) {
    return b ? b->err.c_str() : g_create_err.c_str();
}

// Check that no member was stepped, or had its state replaced, on its own.
static int batch_sync_members(ibpm_batch* b) {
    for (size_t i = 0; i < b->m.size(); ++i) {
        ibpm_handle* h = b->m[i];
        if (h->cur != b->cur)
            return bfail(b, IBPM_ERR_INVALID, "member " + std::to_string(i) +
                                                  " was advanced on its own: batch members must step together");
        if (!h->graphs_ready)  // a changed base flux or transform plan
            return bfail(b, IBPM_ERR_UNSUPPORTED, "member " + std::to_string(i) +
                                                      " changed its base flux, transform plan or level chain "
                                                      "on its own (a batch's are set by ibpm_batch_set_plan "
                                                      "and ibpm_batch_set_chain)");
        b->cold = std::max(b->cold, h->cold);      // set_state on a member re-arms its first steps
    }
    return IBPM_OK;
}

extern "C" int ibpm_batch_advance(ibpm_batch* b, int32_t nsteps) {
    if (!b || nsteps < 0) return IBPM_ERR_INVALID;
    BCK(cudaSetDevice(b->device));
    int rc = batch_sync_members(b);
    if (rc) return rc;
    const int n = (int)b->m.size();
    b->cd.assign((size_t)nsteps * b->off[n], 0.0);
    b->cl.assign((size_t)nsteps * b->off[n], 0.0);
    b->last_steps = nsteps;
    for (auto* h : b->m) BCK(cudaMemsetAsync(h->status, 0, sizeof(int), b->st));
    std::vector<double> hb;
    int done = 0;
    while (done < nsteps) {
        const int k = std::min(b->hist_cap, nsteps - done);
        for (auto* h : b->m) BCK(cudaMemsetAsync(h->counter, 0, sizeof(int), b->st));
        for (int s = 0; s < k; ++s) BCK(batch_step(b));
        for (int i = 0; i < n; ++i) {
            ibpm_handle* h = b->m[i];
            hb.resize((size_t)k * 2 * h->nbodies);
            BCK(cudaMemcpyAsync(hb.data(), h->hist, sizeof(double) * hb.size(), cudaMemcpyDeviceToHost, b->st));
            BCK(cudaStreamSynchronize(b->st));
            for (int s = 0; s < k; ++s)
                for (int j = 0; j < h->nbodies; ++j) {
                    const size_t o = ((size_t)(done + s)) * b->off[n] + b->off[i] + j;
                    b->cd[o] = hb[((size_t)s * 2 + 0) * h->nbodies + j];
                    b->cl[o] = hb[((size_t)s * 2 + 1) * h->nbodies + j];
                }
        }
        done += k;
    }
    BCK(cudaStreamSynchronize(b->st));
    for (size_t i = 0; i < b->m.size(); ++i) {
        int hs = 0;
        BCK(cudaMemcpy(&hs, b->m[i]->status, sizeof(int), cudaMemcpyDeviceToHost));
        if (hs & 8) return bfail(b, IBPM_ERR_CUDA, "member " + std::to_string(i) + ": internal: a step ran past the force history");
        if (hs) return bfail(b, IBPM_ERR_NONFINITE, "member " + std::to_string(i) + ": CD/CL became non-finite");
    }
    return IBPM_OK;
}

extern "C" int ibpm_batch_get_forces(const ibpm_batch* b, int32_t i, double* CD, double* CL) {
    if (!b || i < 0 || i >= (int)b->m.size()) return IBPM_ERR_INVALID;
    const int nb = b->m[i]->nbodies, tot = b->off.back();
    for (int s = 0; s < b->last_steps; ++s)
        for (int j = 0; j < nb; ++j) {
            if (CD) CD[(size_t)s * nb + j] = b->cd[(size_t)s * tot + b->off[i] + j];
            if (CL) CL[(size_t)s * nb + j] = b->cl[(size_t)s * tot + b->off[i] + j];
        }
    return IBPM_OK;
}

extern "C" int ibpm_batch_bench(ibpm_batch* b, int32_t nsteps, int32_t flush_l2, double* step_ms) {
    if (!b || nsteps < 1 || !step_ms) return IBPM_ERR_INVALID;
    BCK(cudaSetDevice(b->device));
    int rc = batch_sync_members(b);
    if (rc) return rc;
    ibpm_handle* h0 = b->m[0];
    if (flush_l2 && !h0->flush_buf) {
        h0->flush_bytes = (size_t)512 << 20;
        if ((rc = dalloc(h0, (char**)&h0->flush_buf, h0->flush_bytes))) return bfail(b, rc, h0->err);
    }
    std::vector<cudaEvent_t> ev(2 * nsteps);
    for (auto& e : ev) BCK(cudaEventCreate(&e));
    int done = 0;
    while (done < nsteps) {
        const int k = std::min(b->hist_cap, nsteps - done);
        for (auto* h : b->m) BCK(cudaMemsetAsync(h->counter, 0, sizeof(int), b->st));
        for (int s = 0; s < k; ++s) {
            if (flush_l2) BCK(cudaMemsetAsync(h0->flush_buf, (done + s) & 0xff, h0->flush_bytes, b->st));
            BCK(cudaEventRecord(ev[2 * (done + s)], b->st));
            BCK(batch_step(b));
            BCK(cudaEventRecord(ev[2 * (done + s) + 1], b->st));
        }
        done += k;
    }
    BCK(cudaStreamSynchronize(b->st));
    for (int s = 0; s < nsteps; ++s) {
        float ms = 0;
        BCK(cudaEventElapsedTime(&ms, ev[2 * s], ev[2 * s + 1]));
        step_ms[s] = ms;
    }
    for (auto& e : ev) cudaEventDestroy(e);
    return IBPM_OK;
}

extern "C" const char* ibpm_kernel_name(int32_t k) {
    return (k >= 0 && k < K_COUNT) ? kKernelNames[k] : "";
}

extern "C" void* ibpm_host_alloc(int64_t bytes) {
    void* p = nullptr;
    if (bytes <= 0 || cudaHostAlloc(&p, (size_t)bytes, cudaHostAllocDefault) != cudaSuccess) return nullptr;
    return p;
}

extern "C" int ibpm_host_free(void* p) {
    if (!p) return IBPM_ERR_INVALID;
    return cudaFreeHost(p) == cudaSuccess ? IBPM_OK : IBPM_ERR_CUDA;
}
