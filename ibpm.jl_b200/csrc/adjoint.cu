// Discrete adjoint of the static-body IBPM step: the transpose of the
// derivative of advance!(state, prob, t) (src/timestepping/timestepping.jl:35-67),
// one operator at a time.  Every kernel is written in gather form (each output
// element sums its own inputs in a fixed order), so the adjoint is
// deterministic like the forward step.  Index comments use 0-based indices:
// Γ-like (i, j) with i < nx-1, j < ny-1; fluxes qx[I, J] (I ≤ nx, J < ny) and
// qy[I, J] (I < nx, J ≤ ny) at I + J(nx+1) and nu + I + J nx; edge vectors with
// the reference's LEFT/RIGHT/BOT/TOP segment offsets (fluid-domain.jl:68-69).
#include "ibpm_internal.cuh"

namespace ibpm {

// Value of entry e of an edge vector that the previous (finer) level of the
// adjoint level chain produced: its curl part (bc, may be null) plus the
// transpose of apply_bc!(·, ψbc, 1) applied to its solve result W (may be
// null): the edge rows/columns of W (mg-utils.jl:43-60).
struct EdgeAdj {
    const double* bc;
    const double* W;
    __device__ double operator()(const Geom& g, int e) const {
        double v = bc ? bc[e] : 0.0;
        if (W) {
            const int P = g.P, n1 = g.n1, n2 = g.n2;
            if (e >= g.B && e < g.T) {
                const int u = e - g.B;
                if (u >= 1 && u <= n1) v += W[u - 1];
            } else if (e >= g.T) {
                const int u = e - g.T;
                if (u >= 1 && u <= n1) v += W[(long long)(n2 - 1) * P + u - 1];
            } else if (e < g.R) {
                const int u = e - g.L;
                if (u >= 1 && u <= n2) v += W[(long long)(u - 1) * P];
            } else {
                const int u = e - g.R;
                if (u >= 1 && u <= n2) v += W[(long long)(u - 1) * P + n1 - 1];
            }
        }
        return v;
    }
};

// Transpose of get_bc! (mg-utils.jl:7-32) at the coarse point (i, j): each
// sample line takes its even edge entry with weight 1 and the odd entries on
// either side with weight ½.
template <class BV>
__device__ double get_bc_T_at(const Geom& g, int i, int j, const BV& b) {
    const int nx = g.nx, ny = g.ny;
    double v = 0.0;
    auto line = [&](int seg, int m, int half) {
        if (m < 0 || m > half) return;
        v += b(g, seg + 2 * m);
        if (m >= 1) v += 0.5 * b(g, seg + 2 * m - 1);
        if (m + 1 <= half) v += 0.5 * b(g, seg + 2 * m + 1);
    };
    if (j == ny / 4 - 1) line(g.B, i - nx / 4 + 1, nx / 2);
    if (j == 3 * ny / 4 - 1) line(g.T, i - nx / 4 + 1, nx / 2);
    if (i == nx / 4 - 1) line(g.L, j - ny / 4 + 1, ny / 2);
    if (i == 3 * nx / 4 - 1) line(g.R, j - ny / 4 + 1, ny / 2);
    return v;
}

// ---------------------------------------------------------------------------
// Adjoint level chain of vort2flux! (curl.jl:147-162), one level:
//   ψ̄ = rot(q̄) + get_bc!ᵀ(b̄_prev)      (the interior of curl! is rot!ᵀ)
//   bc_out = the edge part of curl!ᵀ(q̄), with its bottom row at ψbc[(B-1)+i]
// Threads [0, nΓ) write ψ̄, threads [nΓ, nΓ + nbc) write bc_out.
// ---------------------------------------------------------------------------
__global__ void adj_curlT_kernel(Geom g, const double* __restrict__ qb, EdgeAdj prev, double* psib,
                                 double* bc_out) {
    pdl_wait();
    pdl_trigger();
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int nx = g.nx, ny = g.ny, n1 = g.n1, n2 = g.n2;
    const int nG = n1 * n2;
    auto qx = [&](int I, int J) -> double { return qb ? qb[I + (long long)J * (nx + 1)] : 0.0; };
    auto qy = [&](int I, int J) -> double { return qb ? qb[g.nu + I + (long long)J * nx] : 0.0; };
    if (t < nG) {
        const int i = t % n1, j = t / n1;
        double v = ((qx(i + 1, j) - qx(i + 1, j + 1)) + qy(i + 1, j + 1)) - qy(i, j + 1);
        if (prev.bc || prev.W) v += get_bc_T_at(g, i, j, prev);
        psib[(long long)j * g.P + i] = v;
    } else if (t < nG + g.nbc) {
        const int e = t - nG;
        double v = 0.0;
        if (e < g.R) {                                  // LEFT, v = 0 … ny
            const int u = e - g.L;
            if (u >= 1) v += qx(0, u - 1);
            if (u <= ny - 1) v -= qx(0, u);
            if (u >= 1 && u <= ny - 1) v += qy(0, u);
        } else if (e < g.B) {                           // RIGHT
            const int u = e - g.R;
            if (u >= 1) v += qx(nx, u - 1);
            if (u <= ny - 1) v -= qx(nx, u);
            if (u >= 1 && u <= ny - 1) v -= qy(nx - 1, u);
        } else if (e < g.T) {                           // BOT, u = 0 … nx
            const int u = e - g.B;
            if (u <= nx - 2) v -= qx(u + 1, 0);
            if (u <= nx - 1) v += qy(u, 0);
            if (u >= 1) v -= qy(u - 1, 0);
        } else {                                        // TOP
            const int u = e - g.T;
            if (u >= 1 && u <= nx - 1) v += qx(u, ny - 1);
            if (u <= nx - 1) v += qy(u, ny);
            if (u >= 1) v -= qy(u - 1, ny);
        }
        bc_out[e] = v;
    }
}

cudaError_t launch_adj_curlT(const Geom& g, const double* qb, const double* prev_bc, const double* prev_W,
                             double* psib, double* bc_out, cudaStream_t st) {
    const int n = g.n1 * g.n2 + g.nbc;
    EdgeAdj prev{prev_bc, prev_W};
    return launch_k(adj_curlT_kernel, dim3((n + 255) / 256), dim3(256), 0, st, g, qb, prev, psib, bc_out);
}

// ---------------------------------------------------------------------------
// Transpose of one coarsify! (mg-utils.jl:71-106): level `lev`'s centre was
// overwritten with the full-weighting restriction of level lev-1, so every
// point of level lev-1 gathers its weight (1, ½ or ¼) of the centre adjoints
// whose 3×3 stencil holds it.  blockIdx.z = 1 clears the centre of level
// `zero_lev` (an earlier link of the chain already moved it down).
// ---------------------------------------------------------------------------
__global__ void adj_coarsifyT_kernel(Geom g, double* G, long long lstride, int lev, int zero_lev) {
    pdl_wait();
    pdl_trigger();
    const int nx = g.nx, ny = g.ny, P = g.P;
    if (blockIdx.z == 1) {
        const int na = nx / 2 - 1, nb = ny / 2 - 1;
        const int t = blockIdx.x * blockDim.x + threadIdx.x;
        if (t >= na * nb) return;
        const int a = t % na, b = t / na;
        G[(long long)zero_lev * lstride + (long long)(ny / 4 + b) * P + nx / 4 + a] = 0.0;
        return;
    }
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= g.n1 * g.n2) return;
    const int i = t % g.n1, j = t / g.n1;
    const double* C = G + (long long)lev * lstride;
    int ai[2], na = 0, bj[2], nb = 0;
    double wi[2], wj[2];
    // centre point a sits at fine index 2a+1; 0 <= a < nx/2 - 1
    if (i & 1) { ai[na] = (i - 1) / 2; wi[na++] = 1.0; }
    else {
        if (i >= 2) { ai[na] = (i - 2) / 2; wi[na++] = 0.5; }
        ai[na] = i / 2; wi[na++] = 0.5;
    }
    if (j & 1) { bj[nb] = (j - 1) / 2; wj[nb++] = 1.0; }
    else {
        if (j >= 2) { bj[nb] = (j - 2) / 2; wj[nb++] = 0.5; }
        bj[nb] = j / 2; wj[nb++] = 0.5;
    }
    double v = 0.0;
    for (int p = 0; p < na; ++p) {
        if (ai[p] > nx / 2 - 2) continue;
        for (int r = 0; r < nb; ++r) {
            if (bj[r] > ny / 2 - 2) continue;
            v += (wi[p] * wj[r]) * C[(long long)(ny / 4 + bj[r]) * P + nx / 4 + ai[p]];
        }
    }
    G[(long long)(lev - 1) * lstride + (long long)j * P + i] += v;
}

cudaError_t launch_adj_coarsifyT(const Geom& g, double* G, long long lstride, int lev, int zero_lev,
                                 cudaStream_t st) {
    const int n = g.n1 * g.n2;
    dim3 grid((n + 255) / 256, 1, zero_lev >= 0 ? 2 : 1);
    return launch_k(adj_coarsifyT_kernel, grid, dim3(256), 0, st, g, G, lstride, lev, zero_lev);
}

__global__ void zero_centre_kernel(Geom g, double* G) {
    pdl_wait();
    pdl_trigger();
    const int na = g.nx / 2 - 1, nb = g.ny / 2 - 1;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= na * nb) return;
    G[(long long)(g.ny / 4 + t / na) * g.P + g.nx / 4 + t % na] = 0.0;
}

cudaError_t launch_zero_centre(const Geom& g, double* G, cudaStream_t st) {
    const int n = (g.nx / 2 - 1) * (g.ny / 2 - 1);
    return launch_k(zero_centre_kernel, dim3((n + 255) / 256), dim3(256), 0, st, g, G);
}

// ---------------------------------------------------------------------------
// Projection adjoint, force side: F̄t = (objective weight of this step) −
// E · rot!ᵀ(W) with W = A⁻¹₁ Γ̄' (transpose of Γ −= A⁻¹ C'E' F̃b,
// timestepping.jl:204-223).  One warp per force component, like E.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__global__ void adj_E_rotT_kernel(BodyDev b, Geom g, const double* __restrict__ W, double wx, double wy,
                                  const double* __restrict__ stepw, const int* __restrict__ adj_n, double* Ft) {
    pdl_wait();
    pdl_trigger();
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= b.nf) return;
    const int kk = warp, comp = kk / b.nb, k = kk % b.nb;
    const int nx = g.nx, ny = g.ny, P = g.P;
    const int bx = b.bidx[k], by = b.bidx[b.nb + k];
    const double* w = b.w + (long long)kk * 169;
    auto Wv = [&](int i, int j) -> double { return W[(long long)j * P + i]; };
    double acc = 0.0;
    for (int t = lane; t < 169; t += 32) {
        const int l = t / 13, m = t % 13;
        const int I = bx + l - 6 - 1, J = by + m - 6 - 1;   // 0-based flux indices
        double qv = 0.0;
        if (comp == 0) {                                  // rot!ᵀ onto qx[I, J]
            if (I >= 1 && I <= nx - 1) {
                if (J <= ny - 2) qv += Wv(I - 1, J);
                if (J >= 1) qv -= Wv(I - 1, J - 1);
            }
        } else {                                          // rot!ᵀ onto qy[I, J]
            if (J >= 1 && J <= ny - 1) {
                if (I >= 1) qv += Wv(I - 1, J - 1);
                if (I <= nx - 2) qv -= Wv(I, J - 1);
            }
        }
        acc += w[t] * qv;
    }
    acc = warp_sum_d(acc);
    if (lane == 0) Ft[kk] = stepw[*adj_n] * (comp == 0 ? wx : wy) - acc;
}

cudaError_t launch_adj_E_rotT(const Geom& g, const BodyDev& b, const double* W, double wx, double wy,
                              const double* stepw, const int* adj_n, double* Ft, cudaStream_t st) {
    const int blocks = (b.nf * 32 + 255) / 256;
    return launch_k(adj_E_rotT_kernel, dim3(blocks), dim3(256), 0, st, b, g, W, wx, wy, stepw, adj_n, Ft);
}

// Position gradient of one adjoint step (the derivation is in the note above
// launch_dweights): one warp per body point, both force components and both
// coordinates; lanes stride the 13×13 window, warp sums in a fixed order, so
// the accumulation is deterministic.  C r̄ is rot!ᵀ of r̄₁, as in adj_E_rotT.
__global__ void adj_xb_kernel(BodyDev b, Geom g, AdjXbArgs a) {
    pdl_wait();
    pdl_trigger();
    const int p = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (p >= b.nb) return;
    const int nx = g.nx, ny = g.ny, P = g.P;
    const int slot = (*a.adj_n) % a.k;
    const double* Fn = a.tapeFb + (long long)slot * b.nf;
    const double* q1 = a.tapeq1 + (long long)slot * g.nq;
    const int bx = b.bidx[p], by = b.bidx[b.nb + p];
    auto Wv = [&](int i, int j) -> double { return a.rb1[(long long)j * P + i]; };
    double gx = 0.0, gy = 0.0;
    for (int comp = 0; comp < 2; ++comp) {
        const int kk = comp * b.nb + p;
        const double fbar = a.Fbar[kk], fn = Fn[kk];
        const double* wd = a.wd + (long long)kk * 338;
        for (int t = lane; t < 169; t += 32) {
            const int l = t / 13, m = t % 13;
            const int I = bx + l - 7, J = by + m - 7;   // 0-based flux indices
            double u, cr = 0.0;
            if (comp == 0) {
                u = q1[I + (long long)J * (nx + 1)] + a.q0x;
                if (I >= 1 && I <= nx - 1) {
                    if (J <= ny - 2) cr += Wv(I - 1, J);
                    if (J >= 1) cr -= Wv(I - 1, J - 1);
                }
            } else {
                u = q1[g.nu + I + (long long)J * nx] + a.q0y;
                if (J >= 1 && J <= ny - 1) {
                    if (I >= 1) cr += Wv(I - 1, J - 1);
                    if (I <= nx - 2) cr -= Wv(I, J - 1);
                }
            }
            const double v = fbar * u - fn * cr;
            gx += wd[t] * v;
            gy += wd[169 + t] * v;
        }
    }
    gx = warp_sum_d(gx);
    gy = warp_sum_d(gy);
    if (lane == 0) {
        a.gxb[p] += gx;
        a.gxb[b.nb + p] += gy;
    }
}

cudaError_t launch_adj_xb(const Geom& g, const BodyDev& b, const AdjXbArgs& a, cudaStream_t st) {
    const int blocks = (b.nb * 32 + 255) / 256;
    return launch_k(adj_xb_kernel, dim3(blocks), dim3(256), 0, st, b, g, a);
}

// y = Aᵀ x, A row-major n×n (the transpose of F̃b = B⁻¹ F): 32 columns per
// block, the rows split over 8 warps, partial sums added in a fixed order.
__global__ void gemv_t_kernel(const double* __restrict__ A, const double* __restrict__ x, double* y, int n) {
    pdl_wait();
    pdl_trigger();
    __shared__ double part[8][32];
    const int c = blockIdx.x * 32 + (threadIdx.x & 31);
    const int w = threadIdx.x >> 5;
    double acc = 0.0;
    if (c < n)
        for (int r = w; r < n; r += 8) acc += A[(long long)r * n + c] * x[r];
    part[w][threadIdx.x & 31] = acc;
    __syncthreads();
    if (w == 0 && c < n) {
        double s = 0.0;
        for (int u = 0; u < 8; ++u) s += part[u][threadIdx.x];
        y[c] = s;
    }
}

cudaError_t launch_gemv_t(const double* A, const double* x, double* y, int n, cudaStream_t st) {
    return launch_k(gemv_t_kernel, dim3((n + 31) / 32), dim3(256), 0, st, A, x, y, n);
}

// q̄s = E' F̄ on the touched level-1 flux points (reg!, interface-coupling.jl:
// 99-119, contributors in ascending component order), and the sums of q̄s over
// the x and y fluxes (the adjoint of the uniform base flux of E(qs + q0)),
// accumulated into acc[0..1].  One block.
__global__ void adj_Et_kernel(BodyDev b, Geom g, const double* __restrict__ Fbar, double* qsb, double* acc) {
    pdl_wait();
    pdl_trigger();
    __shared__ double red[2][1024];
    double sx = 0.0, sy = 0.0;
    for (int r = threadIdx.x; r < b.n_et_rows; r += blockDim.x) {
        double v = 0.0;
        for (int e = b.et_ptr[r]; e < b.et_ptr[r + 1]; ++e) v += b.w[b.et_w[e]] * Fbar[b.et_k[e]];
        const int f = b.et_flux[r];
        qsb[f] = v;
        if (f < g.nu) sx += v;
        else sy += v;
    }
    red[0][threadIdx.x] = sx;
    red[1][threadIdx.x] = sy;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            red[0][threadIdx.x] += red[0][threadIdx.x + s];
            red[1][threadIdx.x] += red[1][threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        acc[0] += red[0][0];
        acc[1] += red[1][0];
    }
}

cudaError_t launch_adj_Et(const Geom& g, const BodyDev& b, const double* Fbar, double* qsb, double* acc,
                          cudaStream_t st) {
    return launch_k(adj_Et_kernel, dim3(1), dim3(1024), 0, st, b, g, Fbar, qsb, acc);
}

// ---------------------------------------------------------------------------
// Trial-step adjoint (get_trial_state!, timestepping.jl:86-129), all levels.
// With r̄ = A⁻¹ Γ̄s (computed before), N̄ = N̄_next + β1 dt r̄ and the forward
// state (Γ_n, q_n) of the step from the tape:
//   f̄ = rot!ᵀ(N̄ / (4hc²))                                 (nonlinear.jl:186-199)
//   Q = avg_flux(q_n + q0)                                  (nonlinear.jl:17-38)
//   Γ̄_n(i,j) = A r̄ + Qy[i+1,j+1](f̄x[i+1,j] + f̄x[i+1,j+1])
//                   − Qx[i+1,j+1](f̄y[i,j+1] + f̄y[i+1,j+1]) + get_bc!ᵀ(b̄c of level−1)
//   b̄c(level) = fac·apply_bc!ᵀ(r̄) + ¼·(edge part of direct_product!ᵀ)
//   Q̄x[I,J] = −Γe'(I−1,J−1)(f̄y[I−1,J] + f̄y[I,J]),  Q̄y[I,J] = Γe(I−1,J−1)(f̄x[I,J−1] + f̄x[I,J])
//   q̄_n = avg_flux!ᵀ(Q̄),   Σq̄0 += 2 Σ Q̄
// where Γe extends Γ_n by ¼ get_bc!(Γ_n[l+1]) below/above and Γe' left/right
// (direct_product_loops!, nonlinear.jl:73-114).
// ---------------------------------------------------------------------------
struct AdjLevel {
    const AdjTrialArgs& a;
    const Geom& g;
    int lev;
    const double* G;           // Γ_n of this level
    const double* q;           // q_n of this level
    const double* r;           // r̄ of this level
    const double* Nin;         // N̄_next of this level
    CoarseBC cb;               // Γ_n of the next coarser level (¼ get_bc! in the products)
    __device__ double Nbar(int i, int j) const {
        const long long o = (long long)j * g.P + i;
        return Nin[o] + a.b1dt * r[o];
    }
    // f̄ = rot!ᵀ(N̄ s), s = 1/(4hc²)
    __device__ double fx(int I, int J) const {
        if (I < 1 || I > g.nx - 1 || J < 0 || J > g.ny - 1) return 0.0;
        double v = 0.0;
        if (J <= g.ny - 2) v += Nbar(I - 1, J);
        if (J >= 1) v -= Nbar(I - 1, J - 1);
        return v * a.nl_scale[lev];
    }
    __device__ double fy(int I, int J) const {
        if (J < 1 || J > g.ny - 1 || I < 0 || I > g.nx - 1) return 0.0;
        double v = 0.0;
        if (I >= 1) v += Nbar(I - 1, J - 1);
        if (I <= g.nx - 2) v -= Nbar(I, J - 1);
        return v * a.nl_scale[lev];
    }
    __device__ double qx(int I, int J) const { return q[I + (long long)J * (g.nx + 1)]; }
    __device__ double qy(int I, int J) const { return q[g.nu + I + (long long)J * g.nx]; }
    __device__ double Qx(int I, int J) const {    // J >= 1
        return ((qx(I, J) + a.q0x[lev]) + qx(I, J - 1)) + a.q0x[lev];
    }
    __device__ double Qy(int I, int J) const {    // I >= 1
        return ((qy(I, J) + a.q0y[lev]) + qy(I - 1, J)) + a.q0y[lev];
    }
    __device__ double Gv(int i, int j) const { return G[(long long)j * g.P + i]; }
    // Γ extended below/above (vertical neighbours of the x-flux products)
    __device__ double Ge(int i, int j) const {
        if (j < 0) return 0.25 * cb.bot(i + 1);
        if (j > g.ny - 2) return 0.25 * cb.top(i + 1);
        return Gv(i, j);
    }
    // Γ extended left/right (horizontal neighbours of the y-flux products)
    __device__ double Gel(int i, int j) const {
        if (i < 0) return 0.25 * cb.left(j + 1);
        if (i > g.nx - 2) return 0.25 * cb.right(j + 1);
        return Gv(i, j);
    }
    __device__ double Qxb(int I, int J) const {   // J in 1 … ny-1
        return -Gel(I - 1, J - 1) * (fy(I - 1, J) + fy(I, J));
    }
    __device__ double Qyb(int I, int J) const {   // I in 1 … nx-1
        return Ge(I - 1, J - 1) * (fx(I, J - 1) + fx(I, J));
    }
};

__device__ AdjLevel adj_level(const AdjTrialArgs& a, const Geom& g, int lev) {
    const int slot = *a.adj_n % a.k;
    const double* G = a.tapeG + (long long)slot * a.tape_gstride;
    AdjLevel L{a, g, lev, G + (long long)lev * g.S, a.tapeq + (long long)slot * a.tape_qstride + (long long)lev * g.nq,
               a.rb + (long long)lev * g.S, a.Nb_in + (long long)lev * g.S, CoarseBC{}};
    L.cb.rc = (lev < a.mg - 1) ? G + (long long)(lev + 1) * g.S : nullptr;
    L.cb.P = g.P; L.cb.nx = g.nx; L.cb.ny = g.ny;
    return L;
}

// b̄c of every level but the coarsest: threads over (level, edge entry).
__global__ void adj_bc_kernel(AdjTrialArgs a, Geom g) {
    pdl_wait();
    pdl_trigger();
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int lev = blockIdx.y;
    if (t >= g.nbc || lev >= a.mg - 1) return;
    const AdjLevel L = adj_level(a, g, lev);
    const int nx = g.nx, ny = g.ny, P = g.P, n1 = g.n1, n2 = g.n2;
    const double fac = a.fac_bc[lev];
    double v = 0.0;
    if (t >= g.B && t < g.T) {
        const int u = t - g.B;
        if (u >= 1 && u <= n1)
            v = fac * L.r[u - 1] + 0.25 * (L.fx(u, 0) * L.Qy(u, 0));
    } else if (t >= g.T) {
        const int u = t - g.T;
        if (u >= 1 && u <= n1)
            v = fac * L.r[(long long)(n2 - 1) * P + u - 1] + 0.25 * (L.fx(u, ny - 1) * L.Qy(u, ny));
    } else if (t < g.R) {
        const int u = t - g.L;
        if (u >= 1 && u <= n2)
            v = fac * L.r[(long long)(u - 1) * P] + 0.25 * (-L.fy(0, u) * L.Qx(0, u));
    } else {
        const int u = t - g.R;
        if (u >= 1 && u <= n2)
            v = fac * L.r[(long long)(u - 1) * P + n1 - 1] + 0.25 * (-L.fy(nx - 1, u) * L.Qx(nx, u));
    }
    a.bcv[(long long)lev * g.nbc + t] = v;
}

// Γ̄_n and N̄ of this state, one thread per Γ point of one level.
__global__ void adj_rhs_kernel(AdjTrialArgs a, Geom g) {
    pdl_wait();
    pdl_trigger();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int lev = blockIdx.z;
    const int n1 = g.n1, n2 = g.n2, P = g.P;
    if (i >= n1 || j >= n2) return;
    const AdjLevel L = adj_level(a, g, lev);
    const long long o = (long long)j * P + i;
    const double* r = L.r;
    const double rc = r[o];
    const double re = (i + 1 < n1) ? r[o + 1] : 0.0;
    const double rw = (i > 0) ? r[o - 1] : 0.0;
    const double rn = (j + 1 < n2) ? r[o + P] : 0.0;
    const double rs = (j > 0) ? r[o - P] : 0.0;
    double v = rc + a.c_lap[lev] * ((((re + rw) + rn) + rs) - 4.0 * rc);   // A r̄ (A is symmetric)
    v += L.Qy(i + 1, j + 1) * (L.fx(i + 1, j) + L.fx(i + 1, j + 1));
    v -= L.Qx(i + 1, j + 1) * (L.fy(i, j + 1) + L.fy(i + 1, j + 1));
    if (lev >= 1) {
        struct {
            const double* bc;
            __device__ double operator()(const Geom&, int e) const { return bc[e]; }
        } bv{a.bcv + (long long)(lev - 1) * g.nbc};
        v += get_bc_T_at(g, i, j, bv);
    }
    const long long go = (long long)lev * g.S + o;
    a.Gb[go] = v;
    a.Nb_out[go] = a.b2dt * rc;
}

// q̄_n = avg_flux!ᵀ(Q̄), one thread per flux element of one level, and the
// per-block partial sums 2ΣQ̄x (J >= 1), 2ΣQ̄y (I >= 1) added to the block's
// own slot of q0part (fixed order over steps).
__global__ void adj_nlq_kernel(AdjTrialArgs a, Geom g) {
    pdl_wait();
    pdl_trigger();
    __shared__ double red[2][256];
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    const int lev = blockIdx.y;
    const int nx = g.nx, ny = g.ny;
    double sx = 0.0, sy = 0.0;
    if (e < g.nq) {
        const AdjLevel L = adj_level(a, g, lev);
        double v = 0.0;
        if (e < g.nu) {
            const int I = e % (nx + 1), J = e / (nx + 1);
            if (J >= 1) {
                const double qb = L.Qxb(I, J);
                v += qb;
                sx = 2.0 * qb;
            }
            if (J + 1 <= ny - 1) v += L.Qxb(I, J + 1);
        } else {
            const int f = e - g.nu;
            const int I = f % nx, J = f / nx;
            if (I >= 1) {
                const double qb = L.Qyb(I, J);
                v += qb;
                sy = 2.0 * qb;
            }
            if (I + 1 <= nx - 1) v += L.Qyb(I + 1, J);
        }
        a.qb[(long long)lev * g.nq + e] = v;
    }
    red[0][threadIdx.x] = sx;
    red[1][threadIdx.x] = sy;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            red[0][threadIdx.x] += red[0][threadIdx.x + s];
            red[1][threadIdx.x] += red[1][threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        double* slot = a.q0part + 2 * ((long long)lev * gridDim.x + blockIdx.x);
        slot[0] += red[0][0];
        slot[1] += red[1][0];
    }
}

int adj_nlq_blocks(const Geom& g) { return (g.nq + 255) / 256; }

cudaError_t launch_adj_trial(const Geom& g, const AdjTrialArgs& a, cudaStream_t st) {
    cudaError_t e;
    if (a.mg > 1 &&
        (e = launch_k(adj_bc_kernel, dim3((g.nbc + 255) / 256, a.mg - 1), dim3(256), 0, st, a, g)) != cudaSuccess)
        return e;
    if ((e = launch_k(adj_rhs_kernel, dim3((g.n1 + 31) / 32, (g.n2 + 7) / 8, a.mg), dim3(32, 8), 0, st, a, g)) !=
        cudaSuccess)
        return e;
    return launch_k(adj_nlq_kernel, dim3(adj_nlq_blocks(g), a.mg), dim3(256), 0, st, a, g);
}

// Step counter of the adjoint sweep (the tape slot and objective weight of
// the kernels above): n ← n − 1 after each adjoint step.
__global__ void adj_tick_kernel(int* adj_n) {
    pdl_wait();
    pdl_trigger();
    *adj_n -= 1;
}

cudaError_t launch_adj_tick(int* adj_n, cudaStream_t st) {
    return launch_k(adj_tick_kernel, dim3(1), dim3(1), 0, st, adj_n);
}

}  // namespace ibpm
