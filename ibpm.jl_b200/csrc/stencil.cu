// Grid stencils of the IBPM step: the right-hand side of the trial solve
// (nonlinear term + AB2 + explicit viscous term + cross-level BCs), coarsify!
// and the multigrid curl.  Index comments use the reference's 1-based
// (Julia) indices; device arrays are 0-based (see ibpm_internal.cuh).
#include "ibpm_internal.cuh"

namespace ibpm {

// ---------------------------------------------------------------------------
// Trial right-hand side, one thread per Γ point of one level:
//   bc   = get_bc!(Γ[lev+1])                   (timestepping.jl:101-106)
//   rhsbc= apply_bc!(0, bc, 0.25 dt/(Re hc²))
//   N    = nonlinear!(Γ, q, q0, 0.25 bc)       (nonlinear.jl:168-201)
//   rhs  = A Γ + β1 dt N + β2 dt Nprev + rhsbc  (timestepping.jl:111-118)
// A Γ is evaluated as the 5-point stencil Γ + c (Σ neighbours − 4Γ), c =
// dt/(2 Re hc²), with zero Dirichlet edges: the operator the reference applies
// through two DSTs with the eigenvalues 1 − Λ c (laplacian.jl:73-76), whose
// eigenvectors are exactly the DST-I basis.
// ---------------------------------------------------------------------------
// LIN: the linearised problem's term (nonlinear.jl:45-65, 144-163),
//   N = C'(DP(Q, ΓB) + DP(QB, Γ)) / (4 hc²),
// Q the face sums of q without base flux, QB those of the base state with its
// base flux, both products using this state's edge values ¼ get_bc!(Γ[l+1])
// (the reference passes the perturbation's Γbc to the ΓB product too).
// MOV: a moving grid's per-face base flux (MovingFlux) instead of q0x, q0y.
// GRP: the simulations of a batch group, blockIdx.z = simulation · mg + level,
// each with its own arguments in ga[simulation] (its fields, coefficients).
template <bool LIN, bool MOV, bool GRP = false>
__global__ void __launch_bounds__(256) trial_rhs_kernel(RhsArgs a0, const RhsArgs* __restrict__ ga, Geom g) {
    pdl_wait();
    pdl_trigger();
    const RhsArgs& a = GRP ? ga[blockIdx.z / g.mg] : a0;
    const int i0 = blockIdx.x * blockDim.x + threadIdx.x;
    const int j0 = blockIdx.y * blockDim.y + threadIdx.y;
    const int lev = GRP ? (int)(blockIdx.z % g.mg) : (int)blockIdx.z;
    const int nx = g.nx, ny = g.ny, n1 = g.n1, n2 = g.n2, P = g.P;
    if (i0 >= n1 || j0 >= n2) return;
    const double* G = a.G + a.Gmap.off(lev);
    const double* q = a.q + (long long)lev * g.nq;
    const double* qy = q + g.nu;
    const double q0x = a.q0x[lev], q0y = a.q0y[lev];
    // moving grid: the base flux varies along y on x-faces and along x on y-faces
    const double* mrow = MOV ? moving_row(a.mv) : nullptr;
    const double hc = MOV ? ldexp(a.mv.h, lev) : 0.0;

    CoarseBC cb;
    cb.rc = (lev < a.mg - 1) ? a.G + a.Gmap.off(lev + 1) : nullptr;
    cb.P = P; cb.nx = nx; cb.ny = ny;

    // Γ extended by the (0.25-scaled) edge values, vertex indices 0 … nx, 0 … ny.
    auto Ge = [&](int vi, int vj) -> double {
        if (vj == 0) return 0.25 * cb.bot(vi);
        if (vj == ny) return 0.25 * cb.top(vi);
        if (vi == 0) return 0.25 * cb.left(vj);
        if (vi == nx) return 0.25 * cb.right(vj);
        return G[(long long)(vj - 1) * P + (vi - 1)];
    };
    auto qxJ = [&](int I, int J) -> double { return q[(I - 1) + (long long)(J - 1) * (nx + 1)]; };
    auto qyJ = [&](int I, int J) -> double { return qy[(I - 1) + (long long)(J - 1) * nx]; };
    // avg_flux (nonlinear.jl:17-38)
    auto q0xJ = [&](int J) -> double {
        if constexpr (MOV) return moving_q0x(a.mv, mrow, J, ny, hc);
        else return q0x;
    };
    auto q0yI = [&](int I) -> double {
        if constexpr (MOV) return moving_q0y(a.mv, mrow, I, nx, hc);
        else return q0y;
    };
    auto QxJ = [&](int I, int J) -> double { return ((qxJ(I, J) + q0xJ(J)) + qxJ(I, J - 1)) + q0xJ(J - 1); };
    auto QyJ = [&](int I, int J) -> double { return ((qyJ(I, J) + q0yI(I)) + qyJ(I - 1, J)) + q0yI(I - 1); };
    // direct_product_loops! (nonlinear.jl:73-114)
    auto fqxJ = [&](int I, int J) -> double { return QyJ(I, J + 1) * Ge(I - 1, J) + QyJ(I, J) * Ge(I - 1, J - 1); };
    auto fqyJ = [&](int I, int J) -> double {
        return -1.0 * (QxJ(I + 1, J) * Ge(I, J - 1) + QxJ(I, J) * Ge(I - 1, J - 1));
    };
    const int i = i0 + 1, j = j0 + 1;  // Julia Γ index
    double N;
    if constexpr (!LIN) {
        // C' fq (rot!, curl.jl:22-34) scaled by 1/(4 hc²)
        N = ((fqxJ(i + 1, j) - fqxJ(i + 1, j + 1)) + (fqyJ(i + 1, j + 1) - fqyJ(i, j + 1))) * a.nl_scale[lev];
    } else {
        const double* GB = a.GB + a.Gmap.off(lev);
        const double* qB = a.qB + (long long)lev * g.nq;
        const double* qBy = qB + g.nu;
        const double q0Bx = a.q0Bx[lev], q0By = a.q0By[lev];
        auto GeB = [&](int vi, int vj) -> double {   // base Γ, this state's edge values
            if (vj == 0 || vj == ny || vi == 0 || vi == nx) return Ge(vi, vj);
            return GB[(long long)(vj - 1) * P + (vi - 1)];
        };
        auto QxL = [&](int I, int J) -> double { return qxJ(I, J) + qxJ(I, J - 1); };
        auto QyL = [&](int I, int J) -> double { return qyJ(I, J) + qyJ(I - 1, J); };
        auto QBx = [&](int I, int J) -> double {
            return ((qB[(I - 1) + (long long)(J - 1) * (nx + 1)] + q0Bx) + qB[(I - 1) + (long long)(J - 2) * (nx + 1)]) + q0Bx;
        };
        auto QBy = [&](int I, int J) -> double {
            return ((qBy[(I - 1) + (long long)(J - 1) * nx] + q0By) + qBy[(I - 2) + (long long)(J - 1) * nx]) + q0By;
        };
        auto fx = [&](int I, int J) -> double {
            return (QyL(I, J + 1) * GeB(I - 1, J) + QyL(I, J) * GeB(I - 1, J - 1)) +
                   (QBy(I, J + 1) * Ge(I - 1, J) + QBy(I, J) * Ge(I - 1, J - 1));
        };
        auto fy = [&](int I, int J) -> double {
            return -1.0 * (QxL(I + 1, J) * GeB(I, J - 1) + QxL(I, J) * GeB(I - 1, J - 1)) +
                   -1.0 * (QBx(I + 1, J) * Ge(I, J - 1) + QBx(I, J) * Ge(I - 1, J - 1));
        };
        N = ((fx(i + 1, j) - fx(i + 1, j + 1)) + (fy(i + 1, j + 1) - fy(i, j + 1))) * a.nl_scale[lev];
    }

    // explicit viscous operator
    const double gc = G[(long long)j0 * P + i0];
    const double ge = (i0 + 1 < n1) ? G[(long long)j0 * P + i0 + 1] : 0.0;
    const double gw = (i0 > 0) ? G[(long long)j0 * P + i0 - 1] : 0.0;
    const double gn = (j0 + 1 < n2) ? G[(long long)(j0 + 1) * P + i0] : 0.0;
    const double gs = (j0 > 0) ? G[(long long)(j0 - 1) * P + i0] : 0.0;
    const double AG = gc + a.c_lap[lev] * ((((ge + gw) + gn) + gs) - 4.0 * gc);

    // apply_bc!(rhsbc = 0, bc, fac) (mg-utils.jl:43-60)
    double rbc = 0.0;
    if (cb.rc) {
        const double fac = a.fac_bc[lev];
        if (j0 == 0) rbc += fac * cb.bot(i0 + 1);
        if (j0 == n2 - 1) rbc += fac * cb.top(i0 + 1);
        if (i0 == 0) rbc += fac * cb.left(j0 + 1);
        if (i0 == n1 - 1) rbc += fac * cb.right(j0 + 1);
    }
    const long long o = a.Gmap.off(lev) + (long long)j0 * P + i0;
    const double Np = a.Nprev[o];
    a.Nnew[o] = N;
    a.rhs[o] = ((AG + a.b1dt * N) + a.b2dt * Np) + rbc;
}

cudaError_t launch_trial_rhs(const Geom& g, const RhsArgs& a, cudaStream_t st) {
    dim3 blk(32, 8);
    dim3 grid((g.n1 + 31) / 32, (g.n2 + 7) / 8, a.mg);
    const RhsArgs* none = nullptr;
    if (a.GB) return launch_k(trial_rhs_kernel<true, false>, grid, blk, 0, st, a, none, g);
    if (a.mv.tab) return launch_k(trial_rhs_kernel<false, true>, grid, blk, 0, st, a, none, g);
    return launch_k(trial_rhs_kernel<false, false>, grid, blk, 0, st, a, none, g);
}

cudaError_t launch_trial_rhs_group(const Geom& g, const RhsArgs& a0, const RhsArgs* ga, int nsim, cudaStream_t st) {
    dim3 blk(32, 8);
    dim3 grid((g.n1 + 31) / 32, (g.n2 + 7) / 8, nsim * g.mg);
    return launch_k(trial_rhs_kernel<false, false, true>, grid, blk, 0, st, a0, ga, g);
}

// ---------------------------------------------------------------------------
// coarsify! (mg-utils.jl:71-106): the centre half of the coarse level gets the
// full-weighting restriction of the fine level, Γc[ic, jc] =
//   Γ[i,j] + ½ (Γ[i+1,j] + Γ[i,j+1] + Γ[i-1,j] + Γ[i,j-1])
//          + ¼ (Γ[i+1,j+1] + Γ[i+1,j-1] + Γ[i-1,j-1] + Γ[i-1,j+1]),
// i = 2:2:nx-2 ↔ ic = nx/4 + i/2.
// ---------------------------------------------------------------------------
__global__ void coarsify_kernel(double* G, SlabMap fmap, SlabMap cmap, Geom g) {
    pdl_wait();
    pdl_trigger();
    const int nxc = g.nx / 2 - 1, nyc = g.ny / 2 - 1;
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    const int b = blockIdx.y * blockDim.y + threadIdx.y;
    if (a >= nxc || b >= nyc) return;
    const int P = g.P;
    const double* F = G + fmap.off(blockIdx.z);
    double* C = G + cmap.off(blockIdx.z);
    const int i = 2 * a + 1, j = 2 * b + 1;  // 0-based fine point
    auto f = [&](int ii, int jj) -> double { return F[(long long)jj * P + ii]; };
    const double e = ((f(i + 1, j) + f(i, j + 1)) + f(i - 1, j)) + f(i, j - 1);
    const double d = ((f(i + 1, j + 1) + f(i + 1, j - 1)) + f(i - 1, j - 1)) + f(i - 1, j + 1);
    C[(long long)(g.ny / 4 + b) * P + (g.nx / 4 + a)] = (f(i, j) + 0.5 * e) + 0.25 * d;
}

cudaError_t launch_coarsify(const Geom& g, double* G, SlabMap fine_map, SlabMap coarse_map, int nslabs,
                            cudaStream_t st) {
    dim3 blk(32, 8);
    dim3 grid((g.nx / 2 - 1 + 31) / 32, (g.ny / 2 - 1 + 7) / 8, nslabs);
    return launch_k(coarsify_kernel, grid, blk, 0, st, G, fine_map, coarse_map, g);
}

// ---------------------------------------------------------------------------
// Multigrid curl (curl.jl:81-116): q = C ψ with edge streamfunction from
// ψbc = get_bc!(ψ[lev+1]) (zero on the coarsest level).  Reproduces the
// reference exactly, including the bottom row of x-fluxes reading ψbc[(B-1)+i]
// (curl.jl:92), i.e. edge vertex i-2, where the top row reads vertex i-1.
// One thread per flux element; blockIdx.y = batch × levels.
// ---------------------------------------------------------------------------
__global__ void curl_kernel(CurlArgs a, Geom g) {
    pdl_wait();
    pdl_trigger();
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= g.nq) return;
    const int y = blockIdx.y;
    const int lev = a.psi_map.level(y);
    const int bt = a.psi_map.batch(y);
    const int nx = g.nx, ny = g.ny, P = g.P;
    const double* psi = a.psi + a.psi_map.off(y);
    CoarseBC eb;
    eb.rc = (lev < a.mg - 1) ? a.coarse + a.coarse_map.off(y) : nullptr;
    eb.P = P; eb.nx = nx; eb.ny = ny;
    auto ps = [&](int I, int J) -> double { return psi[(long long)(J - 1) * P + (I - 1)]; };
    double v;
    if (e < g.nu) {
        const int I = e % (nx + 1) + 1, J = e / (nx + 1) + 1;
        if (I == 1) v = eb.left(J) - eb.left(J - 1);
        else if (I == nx + 1) v = eb.right(J) - eb.right(J - 1);
        else if (J == 1) v = ps(I - 1, 1) - eb.bot(I - 2);
        else if (J == ny) v = eb.top(I - 1) - ps(I - 1, ny - 1);
        else v = ps(I - 1, J) - ps(I - 1, J - 1);
    } else {
        const int f = e - g.nu;
        const int I = f % nx + 1, J = f / nx + 1;
        if (J == 1) v = eb.bot(I - 1) - eb.bot(I);
        else if (J == ny + 1) v = eb.top(I - 1) - eb.top(I);
        else if (I == 1) v = eb.left(J - 1) - ps(1, J - 1);
        else if (I == nx) v = ps(nx - 1, J - 1) - eb.right(J - 1);
        else v = ps(I - 1, J - 1) - ps(I, J - 1);
    }
    a.q[(long long)bt * a.q_bstride + (long long)(lev - a.q_lev0) * a.q_lstride + e] = v;
}

cudaError_t launch_curl(const Geom& g, const CurlArgs& a, cudaStream_t st) {
    dim3 grid((g.nq + 255) / 256, a.nlev * a.nbatch);
    return launch_k(curl_kernel, grid, dim3(256), 0, st, a, g);
}

// ---------------------------------------------------------------------------
// FP64 residual of one refinement sweep of vort2flux! on every level at once,
// stored in FP32 (it is small: the change of ψ since its previous solve):
//     r_ℓ = Γ_ℓ + apply_bc!(get_bc!(ψ_{ℓ+1})) − L ψ_ℓ
// with L x = 4x − Σ neighbours (zero Dirichlet edges), the operator the
// DST-I solve with Λ inverts (laplacian.jl:14-41), and the edge term of a
// level of vort2flux! (curl.jl:151-158, mg-utils.jl:7-60); none at the
// coarsest level.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) resid_lap_kernel(const double* __restrict__ G, const double* __restrict__ psi,
                                                        float* r, Geom g) {
    pdl_wait();
    pdl_trigger();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    // slab z = simulation · mg + level (simulations mg slabs apart)
    const int z = blockIdx.z, lev = z % g.mg;
    const int n1 = g.n1, n2 = g.n2, P = g.P;
    if (i >= n1 || j >= n2) return;
    const double* x = psi + (long long)z * g.S;
    const long long o = (long long)j * P + i;
    const double xc = x[o];
    double nb = 0.0;
    if (i > 0) nb += x[o - 1];
    if (i + 1 < n1) nb += x[o + 1];
    if (j > 0) nb += x[o - P];
    if (j + 1 < n2) nb += x[o + P];
    double v = G[(long long)z * g.S + o];
    if (lev + 1 < g.mg) {
        CoarseBC cb;
        cb.rc = psi + (long long)(z + 1) * g.S; cb.P = P; cb.nx = g.nx; cb.ny = g.ny;
        if (j == 0) v += cb.bot(i + 1);
        if (j == n2 - 1) v += cb.top(i + 1);
        if (i == 0) v += cb.left(j + 1);
        if (i == n1 - 1) v += cb.right(j + 1);
    }
    v -= 4.0 * xc - nb;
    r[(long long)z * g.S + o] = (float)v;
}

cudaError_t launch_resid_lap(const Geom& g, const double* G, const double* psi, float* r, int nsim, cudaStream_t st) {
    dim3 blk(32, 8);
    dim3 grid((g.n1 + 31) / 32, (g.n2 + 7) / 8, g.mg * nsim);
    return launch_k(resid_lap_kernel, grid, blk, 0, st, G, psi, r, g);
}

}  // namespace ibpm
