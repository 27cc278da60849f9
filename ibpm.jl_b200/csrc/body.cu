// Fluid–body coupling of the IBPM step: the regularisation weights of E
// (src/interface-coupling/interface-coupling.jl:6-137), E itself, the
// projection source C'E'F̃b as a deterministic segmented reduction over
// contributions sorted by target, the dense Schur-complement solve and the
// drag/lift reduction (src/timestepping/timestepping.jl:154-163, 204-223,
// 330-354).
#include "ibpm_internal.cuh"

namespace ibpm {

// Yang et al. (2009) smoothed delta function with support ±3 dr, in the
// rounded-coefficient form of interface-coupling.jl:24-61 (result is δ·h).
__device__ double delta_h(double rf, double rb, double dr) {
    const double r = fabs(rf - rb);
    const double r1 = r / dr, r2 = r1 * r1, r3 = r2 * r1, r4 = r3 * r1;
    if (r1 <= 1.0) {
        const double a5 = asin((1.0 / 2.0) * sqrt(3.0) * (2.0 * r1 - 1.0));
        const double a8 = sqrt(1.0 - 12.0 * r2 + 12.0 * r1);
        return 4.166666667e-2 * r4 + (-0.1388888889 + 3.472222222e-2 * a8) * r3 +
               (-7.121664902e-2 - 5.208333333e-2 * a8 + 0.2405626122 * a5) * r2 +
               (-.2405626122 * a5 - 0.3792313933 + 0.1012731481 * a8) * r1 + 8.0187537413e-2 * a5 -
               4.195601852e-2 * a8 + 0.6485698427;
    } else if (r1 <= 2.0) {
        const double a6 = asin((1.0 / 2.0) * sqrt(3.0) * (-3.0 + 2.0 * r1));
        const double a9 = sqrt(-23.0 + 36.0 * r1 - 12.0 * r2);
        return -6.250000000e-2 * r4 + (0.4861111111 - 1.736111111e-2 * a9) * r3 +
               (-1.143175026 + 7.812500000e-2 * a9 - 0.1202813061 * a6) * r2 +
               (0.8751991178 + 0.3608439183 * a6 - 0.1548032407 * a9) * r1 - 0.2806563809 * a6 +
               8.22848104e-3 + 0.1150173611 * a9;
    } else if (r1 <= 3.0) {
        const double a1 = asin((1.0 / 2.0 * (2.0 * r1 - 5.0)) * sqrt(3.0));
        const double a7 = sqrt(-71.0 - 12.0 * r2 + 60.0 * r1);
        return 2.083333333e-2 * r4 + (3.472222222e-3 * a7 - 0.2638888889) * r3 +
               (1.214391675 - 2.604166667e-2 * a7 + 2.405626122e-2 * a1) * r2 +
               (-0.1202813061 * a1 - 2.449273192 + 7.262731481e-2 * a7) * r1 + 0.1523563211 * a1 +
               1.843201677 - 7.306134259e-2 * a7;
    }
    return 0.0;
}

// ∂δh(rf, rb, dr)/∂rb: −sign(rf − rb)/dr times the r1-derivative of the same
// rounded-coefficient pieces (d asin(√3/2 (2r1 − c))/dr1 = √3/√(1 − ¾(2r1 − c)²),
// d √p/dr1 = p'/(2√p)).  At r = 0 the pieces' derivative is ~1e-9 (not exactly
// zero with rounded coefficients); the sign factor makes it 0 there.
__device__ double delta_h_db(double rf, double rb, double dr) {
    const double d = rf - rb;
    const double r1 = fabs(d) / dr, r2 = r1 * r1, r3 = r2 * r1;
    const double s3 = sqrt(3.0);
    double f;
    if (r1 <= 1.0) {
        const double u = 2.0 * r1 - 1.0;
        const double a5 = asin(0.5 * s3 * u), a8 = sqrt(1.0 - 12.0 * r2 + 12.0 * r1);
        const double da5 = s3 / sqrt(1.0 - 0.75 * u * u), da8 = (6.0 - 12.0 * r1) / a8;
        f = 4 * 4.166666667e-2 * r3 + 3 * (-0.1388888889 + 3.472222222e-2 * a8) * r2 + 3.472222222e-2 * da8 * r3 +
            2 * (-7.121664902e-2 - 5.208333333e-2 * a8 + 0.2405626122 * a5) * r1 +
            (-5.208333333e-2 * da8 + 0.2405626122 * da5) * r2 + (-.2405626122 * a5 - 0.3792313933 + 0.1012731481 * a8) +
            (-.2405626122 * da5 + 0.1012731481 * da8) * r1 + 8.0187537413e-2 * da5 - 4.195601852e-2 * da8;
    } else if (r1 <= 2.0) {
        const double u = 2.0 * r1 - 3.0;
        const double a6 = asin(0.5 * s3 * u), a9 = sqrt(-23.0 + 36.0 * r1 - 12.0 * r2);
        const double da6 = s3 / sqrt(1.0 - 0.75 * u * u), da9 = (18.0 - 12.0 * r1) / a9;
        f = -4 * 6.250000000e-2 * r3 + 3 * (0.4861111111 - 1.736111111e-2 * a9) * r2 - 1.736111111e-2 * da9 * r3 +
            2 * (-1.143175026 + 7.812500000e-2 * a9 - 0.1202813061 * a6) * r1 +
            (7.812500000e-2 * da9 - 0.1202813061 * da6) * r2 + (0.8751991178 + 0.3608439183 * a6 - 0.1548032407 * a9) +
            (0.3608439183 * da6 - 0.1548032407 * da9) * r1 - 0.2806563809 * da6 + 0.1150173611 * da9;
    } else if (r1 <= 3.0) {
        const double u = 2.0 * r1 - 5.0;
        const double a1 = asin(0.5 * u * s3), a7 = sqrt(-71.0 - 12.0 * r2 + 60.0 * r1);
        const double da1 = s3 / sqrt(1.0 - 0.75 * u * u), da7 = (30.0 - 12.0 * r1) / a7;
        f = 4 * 2.083333333e-2 * r3 + 3 * (3.472222222e-3 * a7 - 0.2638888889) * r2 + 3.472222222e-3 * da7 * r3 +
            2 * (1.214391675 - 2.604166667e-2 * a7 + 2.405626122e-2 * a1) * r1 +
            (-2.604166667e-2 * da7 + 2.405626122e-2 * da1) * r2 +
            (-0.1202813061 * a1 - 2.449273192 + 7.262731481e-2 * a7) + (-0.1202813061 * da1 + 7.262731481e-2 * da7) * r1 +
            0.1523563211 * da1 - 7.306134259e-2 * da7;
    } else {
        return 0.0;
    }
    const double sg = d > 0.0 ? 1.0 : (d < 0.0 ? -1.0 : 0.0);
    return -sg * f / dr;
}

// Position derivatives of the weights: wd[kk][0][l][m] = ∂w/∂xb_k and
// wd[kk][1][l][m] = ∂w/∂yb_k for the weights of weights_kernel below.
__global__ void dweights_kernel(BodyDev b, double h, double offx, double offy, double* wd) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= b.nf * 169) return;
    const int kk = t / 169, lm = t % 169, l = lm / 13, m = lm % 13;
    const int comp = kk / b.nb, k = kk % b.nb;
    const double xk = b.xb[k], yk = b.xb[b.nb + k];
    const double x = h * (double)((b.bidx[k] - 1) + (l - 6)) - offx + (comp == 1 ? h / 2 : 0.0);
    const double y = h * (double)((b.bidx[b.nb + k] - 1) + (m - 6)) - offy + (comp == 0 ? h / 2 : 0.0);
    wd[(long long)kk * 338 + lm] = delta_h_db(x, xk, h) * delta_h(y, yk, h);
    wd[(long long)kk * 338 + 169 + lm] = delta_h(x, xk, h) * delta_h_db(y, yk, h);
}

cudaError_t launch_dweights(double h, double offx, double offy, const BodyDev& b, double* wd, cudaStream_t st) {
    const int n = b.nf * 169;
    dweights_kernel<<<(n + 255) / 256, 256, 0, st>>>(b, h, offx, offy, wd);
    return cudaGetLastError();
}

// w[kk][l][m], kk = comp·nb + k: weight of flux point (bidx + l − 6, bidx + m − 6)
// for body point k (interface-coupling.jl:89-96).
__global__ void weights_kernel(BodyDev b, double h, double offx, double offy) {
    pdl_wait();
    pdl_trigger();
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= b.nf * 169) return;
    const int kk = t / 169, lm = t % 169, l = lm / 13, m = lm % 13;
    const int comp = kk / b.nb, k = kk % b.nb;
    const double xk = b.xb[k], yk = b.xb[b.nb + k];
    const double x = h * (double)((b.bidx[k] - 1) + (l - 6)) - offx;
    const double y = h * (double)((b.bidx[b.nb + k] - 1) + (m - 6)) - offy;
    double w;
    if (comp == 0) w = delta_h(x, xk, h) * delta_h(y + h / 2, yk, h);
    else w = delta_h(x + h / 2, xk, h) * delta_h(y, yk, h);
    b.w[t] = w;
}

cudaError_t launch_weights(const Geom& g, double h, double offx, double offy, const BodyDev& b,
                           cudaStream_t st) {
    const int n = b.nf * 169;
    weights_kernel<<<(n + 255) / 256, 256, 0, st>>>(b, h, offx, offy);
    return cudaGetLastError();
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// E (regT!, interface-coupling.jl:122-133) on (q + q0): one warp per force
// component and batch member.  F[bt*F_bstride + kk*F_kstride].
// A moving grid's base flux (MovingFlux, level 1) replaces the uniform q0x, q0y.
// Moving bodies: F −= ub·h, the body-point velocity term of boundary_forces!
// (timestepping.jl:174-186), when ub is set.
__global__ void E_kernel(BodyDev b, Geom g, const double* __restrict__ q, long long q_stride, int nbatch,
                         double q0x, double q0y, double* F, long long F_bstride, long long F_kstride,
                         MovingFlux mv, const double* __restrict__ ub, double hub) {
    pdl_wait();
    pdl_trigger();
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= b.nf * nbatch) return;
    const int bt = warp / b.nf, kk = warp % b.nf;
    const int comp = kk / b.nb, k = kk % b.nb;
    const double* qq = q + (long long)bt * q_stride;
    const int bx = b.bidx[k], by = b.bidx[b.nb + k];
    const double* w = b.w + (long long)kk * 169;
    const double* mrow = mv.tab ? moving_row(mv) : nullptr;
    double acc = 0.0;
    for (int t = lane; t < 169; t += 32) {
        const int l = t / 13, m = t % 13;
        const int I = bx + l - 6, J = by + m - 6;
        double qv;
        if (comp == 0)
            qv = qq[(I - 1) + (long long)(J - 1) * (g.nx + 1)] + (mrow ? moving_q0x(mv, mrow, J, g.ny, mv.h) : q0x);
        else
            qv = qq[g.nu + (I - 1) + (long long)(J - 1) * g.nx] + (mrow ? moving_q0y(mv, mrow, I, g.nx, mv.h) : q0y);
        acc += w[t] * qv;
    }
    acc = warp_sum(acc);
    if (ub) acc = acc - ub[kk] * hub;
    if (lane == 0) F[(long long)bt * F_bstride + (long long)kk * F_kstride] = acc;
}

cudaError_t launch_E(const Geom& g, const BodyDev& b, const double* q, long long q_stride, int nbatch,
                     double q0x, double q0y, double* F, long long F_stride, cudaStream_t st,
                     const MovingFlux& mv, const double* ub, double hub) {
    // F_stride > 0: batch stride with unit component stride; F_stride < 0:
    // component stride |F_stride| with unit batch stride (columns of B).
    const long long bs = F_stride > 0 ? F_stride : 1;
    const long long ks = F_stride > 0 ? 1 : -F_stride;
    const long long warps = (long long)b.nf * nbatch;
    const int blocks = (int)((warps * 32 + 255) / 256);
    return launch_k(E_kernel, dim3(blocks), dim3(256), 0, st, b, g, q, q_stride, nbatch, q0x, q0y, F, bs, ks, mv, ub,
                    hub);
}

// y = A x, A row-major n×n: one warp per row (F̃b .= Binv*F̃b, timestepping.jl:160).
__global__ void gemv_kernel(const double* __restrict__ A, const double* __restrict__ x, double* y, int n) {
    pdl_wait();
    pdl_trigger();
    const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (row >= n) return;
    const double* a = A + (long long)row * n;
    double acc = 0.0;
    for (int c = lane; c < n; c += 32) acc += a[c] * x[c];
    acc = warp_sum(acc);
    if (lane == 0) y[row] = acc;
}

cudaError_t launch_gemv(const double* A, const double* x, double* y, int n, cudaStream_t st) {
    return launch_k(gemv_kernel, dim3((n * 32 + 255) / 256), dim3(256), 0, st, A, x, y, n);
}

// update_stress! (timestepping.jl:330-354): fb = F̃b (h/dt) ./ ds,
// CD_j = 2 Σ ds fb_x, CL_j = 2 Σ ds fb_y, written to hist[step][2][nbodies]
// for step < hist_cap (a later step writes nothing and sets bit 3 of *status).
// One block; a non-finite CD/CL sets bit 0 of *status.
__device__ __forceinline__ void stress_block(const BodyDev& b, const double* __restrict__ Fb, double h, double dt,
                                             double* hist, int hist_cap, int* counter, int* status) {
    __shared__ double red[2][256];
    const int step = *counter;
    const bool keep = step >= 0 && step < hist_cap;
    if (!keep && threadIdx.x == 0) atomicOr(status, 8);
    const double hdt = h / dt;
    for (int j = 0; j < b.nbodies; ++j) {
        const int p0 = b.body_start[j], p1 = b.body_start[j + 1];
        double sx = 0.0, sy = 0.0;
        for (int p = p0 + threadIdx.x; p < p1; p += blockDim.x) {
            const double ds = b.ds[p];
            sx += ds * ((Fb[p] * hdt) / ds);
            sy += ds * ((Fb[b.nb + p] * hdt) / ds);
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
            const double cd = 2.0 * red[0][0], cl = 2.0 * red[1][0];
            if (keep) {
                hist[((long long)step * 2 + 0) * b.nbodies + j] = cd;
                hist[((long long)step * 2 + 1) * b.nbodies + j] = cl;
            }
            if (!isfinite(cd) || !isfinite(cl)) atomicOr(status, 1);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) *counter = step + 1;
}

__global__ void stress_kernel(BodyDev b, const double* __restrict__ Fb, double h, double dt, double* hist,
                              int hist_cap, int* counter, int* status) {
    pdl_wait();
    pdl_trigger();
    stress_block(b, Fb, h, dt, hist, hist_cap, counter, status);
}

cudaError_t launch_stress(const BodyDev& b, const double* Fb, double h, double dt, double* hist, int hist_cap,
                          int* counter, int* status, cudaStream_t st) {
    return launch_k(stress_kernel, dim3(1), dim3(256), 0, st, b, Fb, h, dt, hist, hist_cap, counter, status);
}

// Γsrc = C'(E' F̃b) at the Γ points whose rot! stencil touches a regularised
// flux point (timestepping.jl:217, curl.jl:22-34): Γ = (qx₁ − qx₂) +
// (qy₁ − qy₂) over the point's four fluxes, each flux the sum over its sorted
// contributor list (interface-coupling.jl:103-107).  One warp per Γ point:
// the lanes take the contributors of all four fluxes (about 50 at one point
// per h), with the signs of rot!, and a shuffle tree adds them in a fixed
// order, so the result is deterministic (the reference adds sequentially;
// the two agree to round-off).
__device__ __forceinline__ void proj_src_warp(const BodyDev& b, const double* __restrict__ Fb, double* Gsrc, int p,
                                              int lane) {
    if (p >= b.n_src) return;
    double v = 0.0;
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        const int row = b.src_rows[4 * p + r];
        if (row < 0) continue;
        double acc = 0.0;
        for (int e = b.et_ptr[row] + lane; e < b.et_ptr[row + 1]; e += 32) acc += b.w[b.et_w[e]] * Fb[b.et_k[e]];
        v += (r == 0 || r == 2) ? acc : -acc;
    }
    v = warp_sum(v);
    if (lane == 0) Gsrc[b.src_pts[p]] = v;
}

__global__ void proj_src_kernel(BodyDev b, const double* __restrict__ Fb, double* Gsrc) {
    pdl_wait();
    pdl_trigger();
    proj_src_warp(b, Fb, Gsrc, (blockIdx.x * blockDim.x + threadIdx.x) >> 5, threadIdx.x & 31);
}

cudaError_t launch_proj_src(const Geom& g, const BodyDev& b, const double* Fb, double* Gsrc, cudaStream_t st) {
    if (b.n_src == 0) return cudaSuccess;
    const long long threads = (long long)b.n_src * 32;
    return launch_k(proj_src_kernel, dim3((unsigned)((threads + 255) / 256)), dim3(256), 0, st, b, Fb, Gsrc);
}

// update_stress! and the projection source in one launch (both read only F̃b):
// block 0 reduces CD/CL (and advances the step counter), the other blocks
// form C'E'F̃b, one warp per Γ point.
__global__ void stress_src_kernel(BodyDev b, const double* __restrict__ Fb, double h, double dt, double* hist,
                                  int hist_cap, int* counter, int* status, double* Gsrc) {
    pdl_wait();
    pdl_trigger();
    if (blockIdx.x == 0) {
        stress_block(b, Fb, h, dt, hist, hist_cap, counter, status);
        return;
    }
    proj_src_warp(b, Fb, Gsrc, ((blockIdx.x - 1) * blockDim.x + threadIdx.x) >> 5, threadIdx.x & 31);
}

cudaError_t launch_stress_src(const BodyDev& b, const double* Fb, double h, double dt, double* hist, int hist_cap,
                              int* counter, int* status, double* Gsrc, cudaStream_t st) {
    const long long threads = (long long)b.n_src * 32;
    const unsigned blocks = 1 + (unsigned)((threads + 255) / 256);
    return launch_k(stress_src_kernel, dim3(blocks), dim3(256), 0, st, b, Fb, h, dt, hist, hist_cap, counter, status,
                    Gsrc);
}

// C'E' e_kk for unit forces kk = col0 + r (B_times!, laplacian.jl:162), written
// into the level-1 slab of batch member r (slab zeroed beforehand).  One thread
// per point of the 14×14 box of Γ points the 13×13 flux window can reach.
__global__ void unit_src_kernel(BodyDev b, Geom g, int col0, int ncol, double* G, long long bstride) {
    pdl_wait();
    pdl_trigger();
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ncol * 196) return;
    const int r = t / 196, ab = t % 196, da = ab / 14, db = ab % 14;
    const int kk = col0 + r;
    const int comp = kk / b.nb, k = kk % b.nb;
    const int bx = b.bidx[k], by = b.bidx[b.nb + k];
    const double* w = b.w + (long long)kk * 169;
    const int gi = bx - 7 + da, gj = by - 7 + db;  // Julia Γ index
    if (gi < 1 || gi > g.n1 || gj < 1 || gj > g.n2) return;
    auto qx = [&](int I, int J) -> double {
        const int l = I - bx + 6, m = J - by + 6;
        return (comp == 0 && l >= 0 && l < 13 && m >= 0 && m < 13) ? w[l * 13 + m] : 0.0;
    };
    auto qy = [&](int I, int J) -> double {
        const int l = I - bx + 6, m = J - by + 6;
        return (comp == 1 && l >= 0 && l < 13 && m >= 0 && m < 13) ? w[l * 13 + m] : 0.0;
    };
    // Γ[i-1, j-1] = (qx[i, j-1] − qx[i, j]) + (qy[i, j] − qy[i-1, j]), (i, j) = (gi+1, gj+1)
    const double v = (qx(gi + 1, gj) - qx(gi + 1, gj + 1)) + (qy(gi + 1, gj + 1) - qy(gi, gj + 1));
    G[(long long)r * bstride + (long long)(gj - 1) * g.P + (gi - 1)] = v;
}

// ---------------------------------------------------------------------------
// Bodies moved by a MotionFunction (move_body!, move-body-utils.jl:86-133):
// point p of body j at the step's row r = (x, y, cos θ, sin θ, ẋ, ẏ, θ̇) of the
// motion table is xb = (x, y) + Rx x0, ub = (ẋ, ẏ) + Ru x0 with
// Rx = [c −s; s c], Ru = θ̇ [−s −c; c −s], evaluated in the reference's order
// without fused multiply-adds; body_idx = floor((xb + off)/h)
// (interface-coupling.jl:86-87).  A point whose 13×13 window would leave the
// finest grid sets bit 4 of the status word and is clamped inside, so that no
// later kernel reads outside the grid.  The bounding box of the windows'
// centres (min/max body_idx) is accumulated for the projection source.
// ---------------------------------------------------------------------------
__global__ void kinematics_kernel(BodyDev b, Geom g, const double* __restrict__ x0, const double* __restrict__ tab,
                                  const int* __restrict__ step, double h, double offx, double offy, double* xb,
                                  int* bidx, double* ub, int* bbox, int* status) {
    pdl_wait();
    pdl_trigger();
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= b.nb) return;
    int j = 0;
    while (j + 1 < b.nbodies && p >= b.body_start[j + 1]) ++j;
    const double* r = tab + ((long long)(*step) * b.nbodies + j) * 8;
    const double X = x0[p], Y = x0[b.nb + p];
    const double c = r[2], s = r[3], thd = r[6];
    const double xp = __dadd_rn(r[0], __dadd_rn(__dmul_rn(c, X), __dmul_rn(-s, Y)));
    const double yp = __dadd_rn(r[1], __dadd_rn(__dmul_rn(s, X), __dmul_rn(c, Y)));
    xb[p] = xp;
    xb[b.nb + p] = yp;
    ub[p] = __dadd_rn(r[4], __dadd_rn(__dmul_rn(__dmul_rn(thd, -s), X), __dmul_rn(__dmul_rn(thd, -c), Y)));
    ub[b.nb + p] = __dadd_rn(r[5], __dadd_rn(__dmul_rn(__dmul_rn(thd, c), X), __dmul_rn(__dmul_rn(thd, -s), Y)));
    int bx = (int)floor((xp + offx) / h), by = (int)floor((yp + offy) / h);
    if (!(bx - 6 >= 1 && bx + 6 <= g.nx && by - 6 >= 1 && by + 6 <= g.ny)) {
        atomicOr(status, 4);
        bx = min(max(bx, 7), g.nx - 6);
        by = min(max(by, 7), g.ny - 6);
    }
    bidx[p] = bx;
    bidx[b.nb + p] = by;
    atomicMin(&bbox[0], bx);
    atomicMin(&bbox[1], by);
    atomicMax(&bbox[2], bx);
    atomicMax(&bbox[3], by);
}

cudaError_t launch_kinematics(const Geom& g, const BodyDev& b, const double* x0, const double* tab, const int* step,
                              double h, double offx, double offy, double* xb, int* bidx, double* ub, int* bbox,
                              int* status, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(bbox, 0x7f, 2 * sizeof(int), st);   // min slots: a large positive int
    if (e == cudaSuccess) e = cudaMemsetAsync(bbox + 2, 0x80, 2 * sizeof(int), st);  // max slots: a large negative one
    if (e != cudaSuccess) return e;
    return launch_k(kinematics_kernel, dim3((b.nb + 127) / 128), dim3(128), 0, st, b, g, x0, tab, step, h, offx, offy,
                    xb, bidx, ub, bbox, status);
}

// C'E'F̃b on the level-1 slab for moving bodies, every Γ point in gather form:
// each regularised flux sums w·F̃b over the body points whose window holds it,
// in ascending point order (reg!, interface-coupling.jl:99-119), then
// Γ[i-1, j-1] = (qx[i, j-1] − qx[i, j]) + (qy[i, j] − qy[i-1, j]) (rot!).
// Points outside the windows' bounding box are written 0.
__global__ void proj_src_moving_kernel(BodyDev b, Geom g, const double* __restrict__ Fb, const int* __restrict__ bbox,
                                       double* Gsrc) {
    pdl_wait();
    pdl_trigger();
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)g.n1 * g.n2) return;
    const int i0 = (int)(t % g.n1), j0 = (int)(t / g.n1);
    const int i = i0 + 2, j = j0 + 2;  // Julia indices of the fluxes around Γ[i0+1, j0+1]
    double v = 0.0;
    if (i + 1 >= bbox[0] - 6 && i - 1 <= bbox[2] + 6 && j + 1 >= bbox[1] - 6 && j - 1 <= bbox[3] + 6) {
        auto flux = [&](int comp, int I, int J) -> double {
            double q = 0.0;
            for (int k = 0; k < b.nb; ++k) {
                const int l = I - b.bidx[k] + 6, m = J - b.bidx[b.nb + k] + 6;
                if (l >= 0 && l < 13 && m >= 0 && m < 13) {
                    const int kk = comp * b.nb + k;
                    q = __dadd_rn(q, __dmul_rn(b.w[(long long)kk * 169 + l * 13 + m], Fb[kk]));
                }
            }
            return q;
        };
        v = (flux(0, i, j - 1) - flux(0, i, j)) + (flux(1, i, j) - flux(1, i - 1, j));
    }
    Gsrc[(long long)j0 * g.P + i0] = v;
}

cudaError_t launch_proj_src_moving(const Geom& g, const BodyDev& b, const double* Fb, const int* bbox, double* Gsrc,
                                   cudaStream_t st) {
    const long long n = (long long)g.n1 * g.n2;
    return launch_k(proj_src_moving_kernel, dim3((unsigned)((n + 255) / 256)), dim3(256), 0, st, b, g, Fb, bbox, Gsrc);
}

__global__ void info_to_status_kernel(const int* info, int* status) {
    if (*info) atomicOr(status, 2);
}

cudaError_t launch_info_to_status(const int* info, int* status, cudaStream_t st) {
    info_to_status_kernel<<<1, 1, 0, st>>>(info, status);
    return cudaGetLastError();
}

cudaError_t launch_unit_src(const Geom& g, const BodyDev& b, int col0, int ncol, double* G, long long bstride,
                            cudaStream_t st) {
    const int n = ncol * 196;
    unit_src_kernel<<<(n + 255) / 256, 256, 0, st>>>(b, g, col0, ncol, G, bstride);
    return cudaGetLastError();
}

}  // namespace ibpm
