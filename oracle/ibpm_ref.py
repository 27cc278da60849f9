"""FP64 CPU restatement of the static-body IBPM time step of NUFgroup/IBPM.jl.

THIS MODULE IS TEST INFRASTRUCTURE (the oracle). Only ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline legs of ``bench.py`` may
import it, and only as the checker or as the timed CPU baseline. The product
path (``ibpm.jl_b200``) never calls it and has no CPU fallback.

It restates, in numpy/scipy, the algorithm of these reference files (paths are
relative to the IBPM.jl project root):

* ``src/fluid-domain/fluid-domain.jl:44-73``   ``make_grid``
* ``src/fluid-operators/laplacian.jl:14-89``   eigenvalues, Δ⁻¹, A, A⁻¹, B⁻¹
* ``src/fluid-operators/dst-inversion.jl:39-50`` ``dst_inv!``
* ``src/fluid-operators/mg-utils.jl:7-106``      ``get_bc!``, ``apply_bc!``, ``coarsify!``
* ``src/fluid-operators/curl.jl:22-165``        ``rot!``, ``curl!`` (multigrid), ``vort2flux!``
* ``src/fluid-operators/nonlinear.jl:17-201``    ``avg_flux``, ``direct_product!``, ``nonlinear!``
* ``src/interface-coupling/interface-coupling.jl:6-137`` ``δh``, ``setup_reg`` (E, E')
* ``src/timestepping/timestepping.jl:35-354``    ``advance!`` and its helpers
  (``base_flux!`` of a ``MovingGrid``: ``:273-318``)
* ``src/structure-domain/motion-types.jl:40-48`` ``MovingGrid``
* ``src/structure-domain/motion-types.jl:13-17``, ``move-body-utils.jl:86-133``,
  ``timestepping.jl:174-186, 386-398`` ``MotionFunction`` bodies (E and B⁻¹
  rebuilt every step)
* ``src/pre-processing/{models,problem-types,state-types}.jl`` state/problem layout
* ``src/structure-domain/sample-bodies.jl:17-134`` plate, cylinder, NACA bodies

Array convention. A Γ-like field of one level is a 2-D array ``G[i-1, j-1]``
holding the reference's ``Γ[i, j]`` (1-based, column-major, (nx-1)×(ny-1)).
Leading axes (level, batch) are allowed everywhere (``...``).  Fluxes are the
pair ``(qx, qy)`` with shapes (..., nx+1, ny) and (..., nx, ny+1).  The
functions ``*_to_ref``/``*_from_ref`` convert to the reference's flattened
column-major ``(nΓ, mg)`` / ``(nq, mg)`` matrices.

The 2-D DST-I is ``scipy.fft.dstn(type=1)``: unnormalised
``Y_k = 2 Σ_j X_j sin(π (j+1)(k+1)/(n+1))``, the definition of FFTW's RODFT00
that the reference plans in ``dst-inversion.jl:10-20``.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
import scipy.fft as sfft
import scipy.sparse as sp

WORKERS = 1  # scipy.fft worker threads; the timed CPU baseline may raise it


# --------------------------------------------------------------------------
# Grid  (fluid-domain.jl:10-73)
# --------------------------------------------------------------------------
@dataclass
class MultiGrid:
    nx: int
    ny: int
    mg: int
    offx: float
    offy: float
    len: float
    h: float

    @property
    def nGamma(self):
        return (self.nx - 1) * (self.ny - 1)

    @property
    def nu(self):
        return self.ny * (self.nx + 1)

    @property
    def nv(self):
        return self.nx * (self.ny + 1)

    @property
    def nq(self):
        return self.nu + self.nv

    # BC vector offsets, 0-based starts of each segment (fluid-domain.jl:68-69)
    @property
    def LEFT(self):
        return 0

    @property
    def RIGHT(self):
        return self.ny + 1

    @property
    def BOT(self):
        return 2 * (self.ny + 1)

    @property
    def TOP(self):
        return 2 * (self.ny + 1) + self.nx + 1

    @property
    def nbc(self):
        return 2 * (self.nx + 1) + 2 * (self.ny + 1)

    def hc(self, lev):
        """Grid spacing of level ``lev`` (0-based): h·2^lev (timestepping.jl:99)."""
        return self.h * 2 ** lev


def make_grid(h, boundary, mg=1):
    """fluid-domain.jl:44-73. ``boundary`` = (xmin, xmax, ymin, ymax)."""
    offx = -boundary[0]
    offy = -boundary[2]
    ln = boundary[1] - boundary[0]
    ylen = boundary[3] - boundary[2]
    nx = int(round(ln / h))          # Julia round: ties to even, as Python's
    ny = int(round(ylen * nx / ln))
    h = ln / nx
    return MultiGrid(nx=nx, ny=ny, mg=mg, offx=offx, offy=offy, len=ln, h=h)


# --------------------------------------------------------------------------
# Layout conversions to/from the reference's flattened column-major matrices
# --------------------------------------------------------------------------
def gamma_to_ref(G):
    """(mg, nx-1, ny-1) -> (nΓ, mg) column-major as ``state.Γ``."""
    mg = G.shape[0]
    return np.stack([G[l].flatten(order="F") for l in range(mg)], axis=1)


def gamma_from_ref(Gr, g):
    return np.stack([Gr[:, l].reshape((g.nx - 1, g.ny - 1), order="F")
                     for l in range(Gr.shape[1])], axis=0)


def flux_to_ref(qx, qy):
    """(mg, nx+1, ny), (mg, nx, ny+1) -> (nq, mg) as ``state.q``."""
    mg = qx.shape[0]
    return np.stack([np.concatenate([qx[l].flatten(order="F"),
                                     qy[l].flatten(order="F")])
                     for l in range(mg)], axis=1)


def flux_from_ref(qr, g):
    nu = g.nu
    qx = np.stack([qr[:nu, l].reshape((g.nx + 1, g.ny), order="F")
                   for l in range(qr.shape[1])], axis=0)
    qy = np.stack([qr[nu:, l].reshape((g.nx, g.ny + 1), order="F")
                   for l in range(qr.shape[1])], axis=0)
    return qx, qy


# --------------------------------------------------------------------------
# Spectral solves  (laplacian.jl:14-89, dst-inversion.jl:39-50)
# --------------------------------------------------------------------------
def lap_eigs(g):
    """laplacian.jl:14-19: Λ[i,j] = -2(cos(πi/nx) + cos(πj/ny) - 2)."""
    ci = np.cos(np.pi * np.arange(1, g.nx) / g.nx)
    cj = np.cos(np.pi * np.arange(1, g.ny) / g.ny)
    return -2.0 * (ci[:, None] + cj[None, :] - 2.0)


def dst2(x):
    """2-D RODFT00 over the last two axes (dst-inversion.jl:5-8)."""
    return sfft.dstn(x, type=1, axes=(-2, -1), workers=WORKERS)


def dst_inv(b, M, scale):
    """dst-inversion.jl:39-50: x = S((S b) ./ M .* scale)."""
    w = dst2(b)
    w /= M
    w *= scale
    return dst2(w)


def lap_inv_scale(g):
    """The scale 1/(4 nx ny) of get_lap_inv (laplacian.jl:38)."""
    return 1.0 / (4 * g.nx * g.ny)


def ainv_eigs(Lam, dt, Re, hc):
    """get_Ainv (laplacian.jl:61-71): Λ̃ = 1 + Λ dt / (2 Re hc²)."""
    return 1.0 + Lam * dt / (2 * Re * hc ** 2)


def a_eigs(Lam, dt, Re, hc):
    """get_A (laplacian.jl:73-76): the divisor 1 ./ (1 - Λ dt / (2 Re hc²))."""
    return 1.0 / (1.0 - Lam * dt / (2 * Re * hc ** 2))


# --------------------------------------------------------------------------
# Multigrid utilities  (mg-utils.jl)
# --------------------------------------------------------------------------
def get_bc(r, g):
    """mg-utils.jl:7-32: sample the coarse field ``r`` on the fine-grid edge."""
    nx, ny = g.nx, g.ny
    B, T, L, R = g.BOT, g.TOP, g.LEFT, g.RIGHT
    rbc = np.zeros(r.shape[:-2] + (g.nbc,))
    i = nx // 4 + np.arange(0, nx // 2 + 1)           # Julia values (1-based)
    ibc = np.arange(1, nx + 2, 2)
    rbc[..., B + ibc - 1] = r[..., i - 1, ny // 4 - 1]
    rbc[..., T + ibc - 1] = r[..., i - 1, 3 * ny // 4 - 1]
    i = nx // 4 + np.arange(1, nx // 2 + 1)
    ibc = np.arange(2, nx + 1, 2)
    rbc[..., B + ibc - 1] = 0.5 * (r[..., i - 1, ny // 4 - 1] + r[..., i - 2, ny // 4 - 1])
    rbc[..., T + ibc - 1] = 0.5 * (r[..., i - 1, 3 * ny // 4 - 1] + r[..., i - 2, 3 * ny // 4 - 1])
    j = ny // 4 + np.arange(0, ny // 2 + 1)
    jbc = np.arange(1, ny + 2, 2)
    rbc[..., L + jbc - 1] = r[..., nx // 4 - 1, j - 1]
    rbc[..., R + jbc - 1] = r[..., 3 * nx // 4 - 1, j - 1]
    j = ny // 4 + np.arange(1, ny // 2 + 1)
    jbc = np.arange(2, ny + 1, 2)
    rbc[..., L + jbc - 1] = 0.5 * (r[..., nx // 4 - 1, j - 1] + r[..., nx // 4 - 1, j - 2])
    rbc[..., R + jbc - 1] = 0.5 * (r[..., 3 * nx // 4 - 1, j - 1] + r[..., 3 * nx // 4 - 1, j - 2])
    return rbc


def apply_bc(r, rbc, fac, g):
    """mg-utils.jl:43-60, in place: add fac·bc to the edge rows/columns of r."""
    nx, ny = g.nx, g.ny
    B, T, L, R = g.BOT, g.TOP, g.LEFT, g.RIGHT
    fac = np.asarray(fac)[..., None] if np.ndim(fac) else fac
    r[..., :, 0] += fac * rbc[..., B + 1:B + nx]
    r[..., :, ny - 2] += fac * rbc[..., T + 1:T + nx]
    r[..., 0, :] += fac * rbc[..., L + 1:L + ny]
    r[..., nx - 2, :] += fac * rbc[..., R + 1:R + ny]


def coarsify(Gc, G, g):
    """mg-utils.jl:71-106, in place on Gc: fine ``G`` into the coarse centre."""
    nx, ny = g.nx, g.ny
    c = G[..., 1:nx - 2:2, 1:ny - 2:2]                 # Julia i = 2:2:nx-2
    e = (G[..., 2:nx - 1:2, 1:ny - 2:2] + G[..., 1:nx - 2:2, 2:ny - 1:2]
         + G[..., 0:nx - 3:2, 1:ny - 2:2] + G[..., 1:nx - 2:2, 0:ny - 3:2])
    d = (G[..., 2:nx - 1:2, 2:ny - 1:2] + G[..., 2:nx - 1:2, 0:ny - 3:2]
         + G[..., 0:nx - 3:2, 0:ny - 3:2] + G[..., 0:nx - 3:2, 2:ny - 1:2])
    Gc[..., nx // 4:3 * nx // 4 - 1, ny // 4:3 * ny // 4 - 1] = c + 0.5 * e + 0.25 * d


# --------------------------------------------------------------------------
# Curl, rot, vort2flux  (curl.jl)
# --------------------------------------------------------------------------
def rot(qx, qy, g):
    """curl.jl:22-34: Γ = C'q."""
    nx, ny = g.nx, g.ny
    return ((qx[..., 1:nx, 0:ny - 1] - qx[..., 1:nx, 1:ny])
            + (qy[..., 1:nx, 1:ny] - qy[..., 0:nx - 1, 1:ny]))


def curl_mg(psi, psibc, g):
    """curl.jl:81-116: q = Cψ with edge values from ``psibc``.

    Reproduces the reference exactly, including that the bottom row of x-fluxes
    reads ψbc[(B-1)+i] (curl.jl:92) while the top row reads ψbc[T+i] (:371).
    """
    nx, ny = g.nx, g.ny
    B, T, L, R = g.BOT, g.TOP, g.LEFT, g.RIGHT
    lead = psi.shape[:-2]
    qx = np.empty(lead + (nx + 1, ny))
    qy = np.empty(lead + (nx, ny + 1))
    qx[..., 1:nx, 1:ny - 1] = psi[..., :, 1:ny - 1] - psi[..., :, 0:ny - 2]
    qx[..., 1:nx, 0] = psi[..., :, 0] - psibc[..., B:B + nx - 1]
    qx[..., 1:nx, ny - 1] = psibc[..., T + 1:T + nx] - psi[..., :, ny - 2]
    qx[..., 0, :] = psibc[..., L + 1:L + ny + 1] - psibc[..., L:L + ny]
    qx[..., nx, :] = psibc[..., R + 1:R + ny + 1] - psibc[..., R:R + ny]
    qy[..., 1:nx - 1, 1:ny] = psi[..., 0:nx - 2, :] - psi[..., 1:nx - 1, :]
    qy[..., 0, 1:ny] = psibc[..., L + 1:L + ny] - psi[..., 0, :]
    qy[..., nx - 1, 1:ny] = psi[..., nx - 2, :] - psibc[..., R + 1:R + ny]
    qy[..., :, 0] = psibc[..., B:B + nx] - psibc[..., B + 1:B + nx + 1]
    qy[..., :, ny] = psibc[..., T:T + nx] - psibc[..., T + 1:T + nx + 1]
    return qx, qy


def vort2flux(G, Lam, g, mg=None):
    """curl.jl:133-165: multiscale ψ, q from Γ.  Mutates the coarse-level
    centres of ``G`` (coarsify, :419-421) and returns (ψ, qx, qy).

    ``G`` has shape (..., mg, nx-1, ny-1).
    """
    mg = g.mg if mg is None else mg
    for lev in range(1, mg):                                   # :419-421
        coarsify(G[..., lev, :, :], G[..., lev - 1, :, :], g)
    psi = np.zeros_like(G)
    lead = G.shape[:-3]
    qx = np.empty(lead + (mg, g.nx + 1, g.ny))
    qy = np.empty(lead + (mg, g.nx, g.ny + 1))
    scale = lap_inv_scale(g)
    psibc = np.zeros(lead + (g.nbc,))
    psi[..., mg - 1, :, :] = dst_inv(G[..., mg - 1, :, :], Lam, scale)   # :425
    qx[..., mg - 1, :, :], qy[..., mg - 1, :, :] = curl_mg(psi[..., mg - 1, :, :], psibc, g)
    for lev in range(mg - 2, -1, -1):                          # :429-440
        Gwork = G[..., lev, :, :].copy()
        psibc = get_bc(psi[..., lev + 1, :, :], g)
        apply_bc(Gwork, psibc, 1.0, g)
        psi[..., lev, :, :] = dst_inv(Gwork, Lam, scale)
        qx[..., lev, :, :], qy[..., lev, :, :] = curl_mg(psi[..., lev, :, :], psibc, g)
    return psi, qx, qy


# --------------------------------------------------------------------------
# Nonlinear term  (nonlinear.jl)
# --------------------------------------------------------------------------
def avg_flux(qx, qy, q0x, q0y, g):
    """nonlinear.jl:17-38: unscaled 4-face sums Q (edges left at zero)."""
    nx, ny = g.nx, g.ny
    Qx = np.zeros(qx.shape)
    Qy = np.zeros(qy.shape)
    Qx[..., :, 1:ny] = qx[..., :, 1:ny] + q0x[..., :, 1:ny] + qx[..., :, 0:ny - 1] + q0x[..., :, 0:ny - 1]
    Qy[..., 1:nx, :] = qy[..., 1:nx, :] + q0y[..., 1:nx, :] + qy[..., 0:nx - 1, :] + q0y[..., 0:nx - 1, :]
    return Qx, Qy


def direct_product(Qx, Qy, G, Gbc, g):
    """nonlinear.jl:73-114 (with nl_avg! :2-10): fq such that N = C'fq."""
    nx, ny = g.nx, g.ny
    B, T, L, R = g.BOT, g.TOP, g.LEFT, g.RIGHT
    fqx = np.zeros(Qx.shape)
    fqy = np.zeros(Qy.shape)
    fqx[..., 1:nx, 1:ny - 1] = (Qy[..., 1:nx, 2:ny] * G[..., :, 1:ny - 1]
                                + Qy[..., 1:nx, 1:ny - 1] * G[..., :, 0:ny - 2])
    fqx[..., 1:nx, 0] = Qy[..., 1:nx, 1] * G[..., :, 0] + Qy[..., 1:nx, 0] * Gbc[..., B + 1:B + nx]
    fqx[..., 1:nx, ny - 1] = (Qy[..., 1:nx, ny - 1] * G[..., :, ny - 2]
                              + Qy[..., 1:nx, ny] * Gbc[..., T + 1:T + nx])
    fqy[..., 1:nx - 1, 1:ny] = -1.0 * (Qx[..., 2:nx, 1:ny] * G[..., 1:nx - 1, :]
                                       + Qx[..., 1:nx - 1, 1:ny] * G[..., 0:nx - 2, :])
    fqy[..., 0, 1:ny] = -1.0 * (Qx[..., 1, 1:ny] * G[..., 0, :] + Qx[..., 0, 1:ny] * Gbc[..., L + 1:L + ny])
    fqy[..., nx - 1, 1:ny] = -1.0 * (Qx[..., nx - 1, 1:ny] * G[..., nx - 2, :]
                                     + Qx[..., nx, 1:ny] * Gbc[..., R + 1:R + ny])
    return fqx, fqy


def nonlinear(G, qx, qy, q0x, q0y, Gbc_scaled, hc, g):
    """nonlinear.jl:168-201 for one level.  ``Gbc_scaled`` is bc already ×0.25
    (the in-place ``Γbc .*= 0.25`` of :183)."""
    Qx, Qy = avg_flux(qx, qy, q0x, q0y, g)
    fqx, fqy = direct_product(Qx, Qy, G, Gbc_scaled, g)
    N = rot(fqx, fqy, g)
    N *= 1.0 / (4 * hc ** 2)
    return N


def nonlinear_linearized(G, qx, qy, GB, QBx, QBy, Gbc_scaled, hc, g):
    """Linearised term of nonlinear.jl:45-65,144-163: C'(Q⊗ΓB + QB⊗Γ)/(4hc²),
    Q the q-only face sums (no base flux)."""
    zx = np.zeros(qx.shape)
    zy = np.zeros(qy.shape)
    Qx, Qy = avg_flux(qx, qy, zx, zy, g)
    f1x, f1y = direct_product(Qx, Qy, GB, Gbc_scaled, g)
    f2x, f2y = direct_product(QBx, QBy, G, Gbc_scaled, g)
    N = rot(f1x + f2x, f1y + f2y, g)
    N *= 1.0 / (4 * hc ** 2)
    return N


# --------------------------------------------------------------------------
# Interface coupling  (interface-coupling.jl)
# --------------------------------------------------------------------------
def delta_h(rf, rb, dr):
    """interface-coupling.jl:6-62: Yang et al. (2009) smoothed delta (times h),
    support ±3 dr, with the reference's rounded coefficients."""
    r = np.abs(np.asarray(rf, dtype=np.float64) - rb)
    r1 = r / dr
    r2 = r1 * r1
    r3 = r2 * r1
    r4 = r3 * r1
    out = np.zeros_like(r1)
    m1 = r1 <= 1.0
    m2 = (~m1) & (r1 <= 2.0)
    m3 = (~m1) & (~m2) & (r1 <= 3.0)
    if np.any(m1):
        x1, x2, x3, x4 = r1[m1], r2[m1], r3[m1], r4[m1]
        a5 = np.arcsin((1.0 / 2.0) * np.sqrt(3.0) * (2.0 * x1 - 1.0))
        a8 = np.sqrt(1.0 - 12.0 * x2 + 12.0 * x1)
        out[m1] = (4.166666667e-2 * x4 + (-0.1388888889 + 3.472222222e-2 * a8) * x3
                   + (-7.121664902e-2 - 5.208333333e-2 * a8 + 0.2405626122 * a5) * x2
                   + (-.2405626122 * a5 - 0.3792313933 + 0.1012731481 * a8) * x1 + 8.0187537413e-2 * a5
                   - 4.195601852e-2 * a8 + 0.6485698427)
    if np.any(m2):
        x1, x2, x3, x4 = r1[m2], r2[m2], r3[m2], r4[m2]
        a6 = np.arcsin((1.0 / 2.0) * np.sqrt(3.0) * (-3.0 + 2.0 * x1))
        a9 = np.sqrt(-23.0 + 36.0 * x1 - 12.0 * x2)
        out[m2] = (-6.250000000e-2 * x4 + (0.4861111111 - 1.736111111e-2 * a9) * x3
                   + (-1.143175026 + 7.812500000e-2 * a9 - 0.1202813061 * a6) * x2
                   + (0.8751991178 + 0.3608439183 * a6 - 0.1548032407 * a9) * x1 - 0.2806563809 * a6
                   + 8.22848104e-3 + 0.1150173611 * a9)
    if np.any(m3):
        x1, x2, x3, x4 = r1[m3], r2[m3], r3[m3], r4[m3]
        a1 = np.arcsin((1.0 / 2.0 * (2.0 * x1 - 5.0)) * np.sqrt(3.0))
        a7 = np.sqrt(-71.0 - 12.0 * x2 + 60.0 * x1)
        out[m3] = (2.083333333e-2 * x4 + (3.472222222e-3 * a7 - 0.2638888889) * x3
                   + (1.214391675 - 2.604166667e-2 * a7 + 2.405626122e-2 * a1) * x2
                   + (-0.1202813061 * a1 - 2.449273192 + 7.262731481e-2 * a7) * x1 + 0.1523563211 * a1
                   + 1.843201677 - 7.306134259e-2 * a7)
    return out


def delta_h_db(rf, rb, dr):
    """∂δh(rf, rb, dr)/∂rb for delta_h above: −sign(rf − rb)/dr times the
    derivative in r1 = |rf − rb|/dr of the same rounded-coefficient pieces,
    with d asin(√3/2 (2r1 − c))/dr1 = √3 / √(1 − ¾ (2r1 − c)²) and
    d √p(r1)/dr1 = p'(r1) / (2 √p(r1))."""
    d = np.asarray(rf, dtype=np.float64) - rb
    r1 = np.abs(d) / dr
    r2 = r1 * r1
    r3 = r2 * r1
    out = np.zeros_like(r1)
    m1 = r1 <= 1.0
    m2 = (~m1) & (r1 <= 2.0)
    m3 = (~m1) & (~m2) & (r1 <= 3.0)
    s3 = np.sqrt(3.0)
    if np.any(m1):
        x1, x2, x3 = r1[m1], r2[m1], r3[m1]
        u = 2.0 * x1 - 1.0
        a5 = np.arcsin(0.5 * s3 * u)
        a8 = np.sqrt(1.0 - 12.0 * x2 + 12.0 * x1)
        da5 = s3 / np.sqrt(1.0 - 0.75 * u * u)
        da8 = (6.0 - 12.0 * x1) / a8
        out[m1] = (4 * 4.166666667e-2 * x3 + 3 * (-0.1388888889 + 3.472222222e-2 * a8) * x2
                   + 3.472222222e-2 * da8 * x3
                   + 2 * (-7.121664902e-2 - 5.208333333e-2 * a8 + 0.2405626122 * a5) * x1
                   + (-5.208333333e-2 * da8 + 0.2405626122 * da5) * x2
                   + (-.2405626122 * a5 - 0.3792313933 + 0.1012731481 * a8)
                   + (-.2405626122 * da5 + 0.1012731481 * da8) * x1
                   + 8.0187537413e-2 * da5 - 4.195601852e-2 * da8)
    if np.any(m2):
        x1, x2, x3 = r1[m2], r2[m2], r3[m2]
        u = 2.0 * x1 - 3.0
        a6 = np.arcsin(0.5 * s3 * u)
        a9 = np.sqrt(-23.0 + 36.0 * x1 - 12.0 * x2)
        da6 = s3 / np.sqrt(1.0 - 0.75 * u * u)
        da9 = (18.0 - 12.0 * x1) / a9
        out[m2] = (-4 * 6.250000000e-2 * x3 + 3 * (0.4861111111 - 1.736111111e-2 * a9) * x2
                   - 1.736111111e-2 * da9 * x3
                   + 2 * (-1.143175026 + 7.812500000e-2 * a9 - 0.1202813061 * a6) * x1
                   + (7.812500000e-2 * da9 - 0.1202813061 * da6) * x2
                   + (0.8751991178 + 0.3608439183 * a6 - 0.1548032407 * a9)
                   + (0.3608439183 * da6 - 0.1548032407 * da9) * x1
                   - 0.2806563809 * da6 + 0.1150173611 * da9)
    if np.any(m3):
        x1, x2, x3 = r1[m3], r2[m3], r3[m3]
        u = 2.0 * x1 - 5.0
        a1 = np.arcsin(0.5 * u * s3)
        a7 = np.sqrt(-71.0 - 12.0 * x2 + 60.0 * x1)
        da1 = s3 / np.sqrt(1.0 - 0.75 * u * u)
        da7 = (30.0 - 12.0 * x1) / a7
        out[m3] = (4 * 2.083333333e-2 * x3 + 3 * (3.472222222e-3 * a7 - 0.2638888889) * x2
                   + 3.472222222e-3 * da7 * x3
                   + 2 * (1.214391675 - 2.604166667e-2 * a7 + 2.405626122e-2 * a1) * x1
                   + (-2.604166667e-2 * da7 + 2.405626122e-2 * da1) * x2
                   + (-0.1202813061 * a1 - 2.449273192 + 7.262731481e-2 * a7)
                   + (-0.1202813061 * da1 + 7.262731481e-2 * da7) * x1
                   + 0.1523563211 * da1 - 7.306134259e-2 * da7)
    return -np.sign(d) * out / dr


def dE_T(prob, c, qx1, qy1):
    """The position derivative of E contracted with force weights ``c`` (nf,)
    and a level-1 flux v = (qx1, qy1): for every body point p,
    G[p] = Σ_{k ∈ {p, nb+p}} c_k ∂(E v)_k/∂xb_p, shape (nb, 2).  The window
    indices (body_idx) are piecewise constant in xb and the weights vanish at
    the window's edge, so only the δh factors are differentiated."""
    g = prob.grid
    h = g.h
    nb = prob.nb
    s = np.arange(-SUPP, SUPP + 1)
    out = np.zeros((nb, 2))
    for k in range(nb):
        xk, yk = prob.xb[k]
        bx, by = prob.body_idx[k]
        x = h * (bx - 1 + s) - g.offx
        y = h * (by - 1 + s) - g.offy
        I = bx + s - 1                      # 0-based flux indices
        J = by + s - 1
        vx = qx1[np.ix_(I, J)]
        vy = qy1[np.ix_(I, J)]
        # x-force: qx points at (x, y + h/2); y-force: qy points at (x + h/2, y)
        dx1, dy1 = delta_h_db(x, xk, h), delta_h_db(y + h / 2, yk, h)
        fx1, fy1 = delta_h(x, xk, h), delta_h(y + h / 2, yk, h)
        dx2, dy2 = delta_h_db(x + h / 2, xk, h), delta_h_db(y, yk, h)
        fx2, fy2 = delta_h(x + h / 2, xk, h), delta_h(y, yk, h)
        out[k, 0] = (c[k] * np.sum(dx1[:, None] * fy1[None, :] * vx)
                     + c[nb + k] * np.sum(dx2[:, None] * fy2[None, :] * vy))
        out[k, 1] = (c[k] * np.sum(fx1[:, None] * dy1[None, :] * vx)
                     + c[nb + k] * np.sum(fx2[:, None] * dy2[None, :] * vy))
    return out


SUPP = 6


def setup_reg(g, xb):
    """interface-coupling.jl:72-137.  Returns E as a sparse (nf, nq) matrix over
    the reference's flattened level-1 flux vector; E' is its transpose."""
    h = g.h
    nb = xb.shape[0]
    s = np.arange(-SUPP, SUPP + 1)
    bidx = np.empty((nb, 2), dtype=np.int64)
    bidx[:, 0] = np.floor((xb[:, 0] + g.offx) / h).astype(np.int64)   # :86
    bidx[:, 1] = np.floor((xb[:, 1] + g.offy) / h).astype(np.int64)   # :87
    rows, cols, vals = [], [], []
    nxp1 = g.nx + 1
    for k in range(nb):
        x = h * (bidx[k, 0] - 1 + s) - g.offx                          # :91
        y = h * (bidx[k, 1] - 1 + s) - g.offy                          # :92
        w1 = delta_h(x, xb[k, 0], h)[:, None] * delta_h(y + h / 2, xb[k, 1], h)[None, :]
        w2 = delta_h(x + h / 2, xb[k, 0], h)[:, None] * delta_h(y, xb[k, 1], h)[None, :]
        I = bidx[k, 0] + s          # Julia 1-based flux indices
        J = bidx[k, 1] + s
        if I.min() < 1 or J.min() < 1 or I.max() > g.nx or J.max() > g.ny:
            raise ValueError("body point %d: regularisation stencil leaves the grid" % k)
        II, JJ = np.meshgrid(I, J, indexing="ij")
        # qx[i, j] at flat index (i-1) + (j-1)(nx+1)
        rows.append(np.full(II.size, k))
        cols.append(((II - 1) + (JJ - 1) * nxp1).ravel())
        vals.append(w1.ravel())
        # qy[i, j] at nu + (i-1) + (j-1) nx
        rows.append(np.full(II.size, nb + k))
        cols.append((g.nu + (II - 1) + (JJ - 1) * g.nx).ravel())
        vals.append(w2.ravel())
    E = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                      shape=(2 * nb, g.nq))
    return E, bidx


def flux_flat(qx, qy):
    """Single-level (nx+1, ny), (nx, ny+1) -> flat (nq,) in the reference order."""
    lead = qx.shape[:-2]
    return np.concatenate([qx.reshape(lead + (-1,), order="F") if not lead else qx.flatten(order="F"),
                           qy.flatten(order="F") if not lead else qy.reshape(lead + (-1,), order="F")],
                          axis=-1)


def flux_unflat(qf, g):
    qx = qf[:g.nu].reshape((g.nx + 1, g.ny), order="F")
    qy = qf[g.nu:].reshape((g.nx, g.ny + 1), order="F")
    return qx, qy


# --------------------------------------------------------------------------
# Bodies  (sample-bodies.jl)
# --------------------------------------------------------------------------
@dataclass
class Body:
    xb: np.ndarray      # (nb, 2)
    ds: np.ndarray      # (nb,)


def make_cylinder(r, h, x0, y0, n=0):
    """sample-bodies.jl:42-65."""
    circum = 2 * np.pi * r
    if n == 0:
        n = int(math.floor(circum / h / 2))
    step = 2 * np.pi / n
    spt = np.arange(n) * step          # Julia 0:int:(n-1)*int
    xhat = r * np.cos(spt)
    yhat = r * np.sin(spt)
    xb = np.stack([xhat + x0, yhat + y0], axis=1)
    ds = math.sqrt((xhat[1] - xhat[0]) ** 2 + (yhat[1] - yhat[0]) ** 2)
    return Body(xb=xb, ds=np.full(n, ds))


def make_plate(L, alpha, h, x0, y0, n=0):
    """sample-bodies.jl:17-33."""
    if n == 0:
        n = int(math.floor(L / h / 2)) + 1
    spt = L * np.arange(n) / (n - 1)
    xhat = spt * np.cos(-alpha)
    yhat = spt * np.sin(-alpha)
    xb = np.stack([xhat + x0, yhat + y0], axis=1)
    ds = math.sqrt((xhat[1] - xhat[0]) ** 2 + (yhat[1] - yhat[0]) ** 2)
    return Body(xb=xb, ds=np.full(n, ds))


def naca_thickness(x, t):
    """Half-thickness polynomial of sample-bodies.jl:126."""
    return 5 * t * (0.2969 * np.sqrt(x) - 0.1260 * x - 0.3516 * x ** 2 + 0.2843 * x ** 3 - 0.1036 * x ** 4)


def make_naca(x0, N, t, m=0.0, p=0.0, chord=1.0, aoa=0.0, pivot=(0.0, 0.0)):
    """sample-bodies.jl:72-134 with a real-valued thickness ``t`` (the
    reference parses it from a 4-digit string), a chord scale and a rotation
    by ``aoa`` (radians, nose up) about ``pivot``.  Panel midpoints and
    lengths as the reference."""
    dth = np.pi / (N - 1)
    x = 0.5 * (1 + np.cos(dth * np.arange(N)))
    yc = np.zeros_like(x)
    th = np.zeros_like(x)
    if m > 0 and p > 0:
        mi = np.nonzero(x < p)[0][-1]
        yc[:mi + 1] = (m / p ** 2) * (2 * p * x[:mi + 1] - x[:mi + 1] ** 2)
        yc[mi + 1:] = (m / (1 - p) ** 2) * (1 - 2 * p + 2 * p * x[mi + 1:] - x[mi + 1:] ** 2)
        dyc = np.zeros_like(x)
        dyc[:mi + 1] = (2 * m / p ** 2) * (p - x[:mi + 1])
        dyc[mi + 1:] = (2 * m / (1 - p ** 2)) * (p - x[mi + 1:])
        th = np.arctan(dyc)
    yt = naca_thickness(x, t)
    xU = x - yt * np.sin(th)
    yU = yc + yt * np.cos(th)
    yL = yc - yt * np.cos(th)
    xe = np.zeros((2 * N - 1, 2))
    for i in range(N):
        xe[i] = [x[i] - x0, yU[i]]
    for i in range(N - 1):
        xe[i + N] = [x[N - 2 - i] - x0, yL[N - 2 - i]]
    xe *= chord
    if aoa != 0.0:
        c, s_ = math.cos(-aoa), math.sin(-aoa)
        px, py = pivot
        X = xe[:, 0] - px
        Y = xe[:, 1] - py
        xe = np.stack([c * X - s_ * Y + px, s_ * X + c * Y + py], axis=1)
    xb = (xe[1:] + xe[:-1]) / 2.0
    ds = np.sqrt(np.sum((xe[1:] - xe[:-1]) ** 2, axis=1))
    return Body(xb=xb, ds=ds)


# --------------------------------------------------------------------------
# Problem, state and the time step
# --------------------------------------------------------------------------
@dataclass
class MovingGrid:
    """MovingGrid (motion-types.jl:40-48): the grid moves with the body; the
    lab-frame free stream (U(t), V(t)) and the body frame's angular position
    θ(t) (minus the aerodynamic pitch) and rate θ̇(t), all callables of t."""
    U: object
    V: object
    theta: object
    theta_dot: object
    xc: float = 0.0
    yc: float = 0.0


@dataclass
class MotionFunction:
    """MotionFunction (motion-types.jl:13-17): the body's reference points x0
    move rigidly with the frame xc(t) = (x, y, θ) and velocity
    uc(t) = (ẋ, ẏ, θ̇), each a triple of callables."""
    xc: tuple
    uc: tuple


def rigid_motion(m, x0, t):
    """move_body! for a MotionFunction (move-body-utils.jl:86-133): xb = pos +
    Rx x0 and ub = vel + Ru x0 with Rx = [c −s; s c], Ru = θ̇ [−s −c; c −s]."""
    x, y, th = (float(f(t)) for f in m.xc)
    xd, yd, thd = (float(f(t)) for f in m.uc)
    c, s = math.cos(th), math.sin(th)
    X, Y = x0[:, 0], x0[:, 1]
    xb = np.stack([x + (c * X + (-s) * Y), y + (s * X + c * Y)], axis=1)
    ub = np.stack([xd + ((thd * (-s)) * X + (thd * (-c)) * Y), yd + ((thd * c) * X + (thd * (-s)) * Y)], axis=1)
    return xb, ub


def moving_grid_coords(g, xc, yc):
    """models.jl:135-153: per level, y − yc of every x-flux row (YY, shape
    (mg, ny)) and x − xc of every y-flux column (XX, shape (mg, nx)); the
    reference stores them expanded to every flux point."""
    XX = np.zeros((g.mg, g.nx))
    YY = np.zeros((g.mg, g.ny))
    for lev in range(g.mg):
        hc = g.hc(lev)
        y = ((np.arange(1, g.ny + 1) - 0.5) - g.ny / 2) * hc + (g.ny / 2) * g.h - g.offy
        YY[lev] = y - yc
        x = ((np.arange(1, g.nx + 1) - 0.5) - g.nx / 2) * hc + (g.nx / 2) * g.h - g.offx
        XX[lev] = x - xc
    return XX, YY


def moving_grid_rates(prob, t):
    """The scalars of base_flux! for a MovingGrid (timestepping.jl:283-296):
    Ω = −θ̇(t) and the body-frame translation (Ux0, Uy0) of the motion's free
    stream rotated by α = −θ(t), plus the problem's own free stream."""
    m = prob.motion
    Om = -m.theta_dot(t)
    a = -m.theta(t)
    U, V = m.U(t), m.V(t)
    Ux0 = U * math.cos(a) - V * math.sin(a)
    Uy0 = U * math.sin(a) + V * math.cos(a)
    af = prob.inclination
    Ux0 += prob.Ux * math.cos(af) - prob.Uy * math.sin(af)
    Uy0 += prob.Ux * math.sin(af) + prob.Uy * math.cos(af)
    return Om, Ux0, Uy0


@dataclass
class IBProblem:
    """problem-types.jl:23-41 + models.jl:27-159 for Static bodies."""
    grid: MultiGrid
    bodies: list
    dt: float
    Re: float
    Ux: float = 1.0
    Uy: float = 0.0
    inclination: float = 0.0
    beta: tuple = (1.5, -0.5)                   # AB2, models.jl:70-72
    build_binv: bool = True
    Lam: np.ndarray = field(init=False)
    A_M: np.ndarray = field(init=False)         # divisor of A per level
    Ainv_M: np.ndarray = field(init=False)      # divisor of A⁻¹ per level
    E: object = field(init=False)
    B: np.ndarray = field(init=False, default=None)
    Binv: np.ndarray = field(init=False, default=None)
    # LinearizedIBProblem (problem-types.jl:47-87): base Γ and averaged base
    # flux QB per level, or None for the nonlinear problem
    base: tuple = field(init=False, default=None)
    # the bodies' motion: None (Static) or a MovingGrid; xc, yc are the
    # IBModel keywords (models.jl:127-129), which IBProblem never sets, so the
    # rotational flux is taken about (0, 0) whatever MovingGrid.xc/yc say
    motion: object = None
    xc: float = 0.0
    yc: float = 0.0

    def __post_init__(self):
        g = self.grid
        self.Lam = lap_eigs(g)
        self.A_M = np.stack([a_eigs(self.Lam, self.dt, self.Re, g.hc(l)) for l in range(g.mg)])
        self.Ainv_M = np.stack([ainv_eigs(self.Lam, self.dt, self.Re, g.hc(l)) for l in range(g.mg)])
        self.xb = np.concatenate([b.xb for b in self.bodies], axis=0)
        self.nb_list = [b.xb.shape[0] for b in self.bodies]
        self.E, self.body_idx = setup_reg(g, self.xb)
        self.ET = self.E.T.tocsr()
        if self.build_binv:
            self.B = build_B(self)
            self.Binv = np.linalg.inv(self.B)     # laplacian.jl:118 (LAPACK getrf/getri)
        if isinstance(self.motion, MovingGrid):
            assert len(self.bodies) == 1          # models.jl:137, timestepping.jl:277
            self.XX, self.YY = moving_grid_coords(g, self.xc, self.yc)
        if self.moving_bodies:
            assert len(self.motion) == len(self.bodies)
            self.x0 = [b.xb.copy() for b in self.bodies]  # the reference configuration
            self.ub = np.zeros((self.nb, 2))

    @property
    def moving_bodies(self):
        """Every body carries a MotionFunction (MotionType(bodies), move-body-utils.jl:19-26)."""
        return isinstance(self.motion, (list, tuple)) and all(isinstance(m, MotionFunction) for m in self.motion)

    def move_bodies(self, t):
        """update_bodies! for MotionFunction bodies (timestepping.jl:386-398): move
        every body to t, then rebuild E and B⁻¹.  The reference solves with B by
        conjugate gradients to reltol 1e-12 (laplacian.jl:123-141); here B⁻¹ is
        the exact inverse of the rebuilt B, as for static bodies."""
        xbs, ubs = [], []
        for m, x0 in zip(self.motion, self.x0):
            xb, ub = rigid_motion(m, x0, t)
            xbs.append(xb)
            ubs.append(ub)
        self.xb = np.concatenate(xbs, axis=0)
        self.ub = np.concatenate(ubs, axis=0)
        for b, xb in zip(self.bodies, xbs):
            b.xb = xb
        self.E, self.body_idx = setup_reg(self.grid, self.xb)
        self.ET = self.E.T.tocsr()
        if self.build_binv:
            self.B = build_B(self)
            self.Binv = np.linalg.inv(self.B)

    @property
    def nb(self):
        return self.xb.shape[0]

    @property
    def nf(self):
        return 2 * self.nb


def ainv_level(b, prob, lev):
    g = prob.grid
    return dst_inv(b, prob.Ainv_M[lev], lap_inv_scale(g))


def a_level(b, prob, lev):
    g = prob.grid
    return dst_inv(b, prob.A_M[lev], lap_inv_scale(g))


def ECt(fb, prob):
    """(E C)' fb = C'(E' fb) on level 1 (timestepping.jl:217).  ``fb`` may be
    (nf,) or (nf, R); returns (nx-1, ny-1) or (R, nx-1, ny-1)."""
    g = prob.grid
    qf = prob.ET @ fb
    if qf.ndim == 1:
        qx, qy = flux_unflat(qf, g)
        return rot(qx, qy, g)
    R = qf.shape[1]
    qx = qf[:g.nu].T.reshape((R, g.ny, g.nx + 1)).transpose(0, 2, 1)
    qy = qf[g.nu:].T.reshape((R, g.ny + 1, g.nx)).transpose(0, 2, 1)
    return rot(qx, qy, g)


def E_apply(qx1, qy1, prob):
    """E acting on one level-1 flux field (interface-coupling.jl:122-133)."""
    lead = qx1.shape[:-2]
    if not lead:
        return prob.E @ np.concatenate([qx1.flatten(order="F"), qy1.flatten(order="F")])
    R = int(np.prod(lead))
    qxf = qx1.reshape((R,) + qx1.shape[-2:]).transpose(0, 2, 1).reshape(R, -1)
    qyf = qy1.reshape((R,) + qy1.shape[-2:]).transpose(0, 2, 1).reshape(R, -1)
    return (prob.E @ np.concatenate([qxf, qyf], axis=1).T).T.reshape(lead + (-1,))


def B_times(prob, Z):
    """B_times! (laplacian.jl:143-169) of the columns of Z (nf, R):
    E · vort2flux(A⁻¹_1 · C'E' z)[level-1 flux] for each column z."""
    g = prob.grid
    R = Z.shape[1]
    G = np.zeros((R, g.mg, g.nx - 1, g.ny - 1))
    G[:, 0] = ainv_level(ECt(Z, prob), prob, 0)
    _, qx, qy = vort2flux(G, prob.Lam, g)
    return E_apply(qx[:, 0], qy[:, 0], prob).T


def build_B(prob, chunk=64):
    """get_Binv (laplacian.jl:98-119): column j of B is B_times!(e_j), computed
    ``chunk`` columns at a time (the columns are independent)."""
    nf = prob.nf
    B = np.zeros((nf, nf))
    for c0 in range(0, nf, chunk):
        c1 = min(nf, c0 + chunk)
        Z = np.zeros((nf, c1 - c0))
        Z[np.arange(c0, c1), np.arange(c1 - c0)] = 1.0
        B[:, c0:c1] = B_times(prob, Z)
    return B


@dataclass
class IBState:
    """state-types.jl:7-47 (the fields the static step uses)."""
    Gamma: np.ndarray          # (mg, nx-1, ny-1)
    psi: np.ndarray
    qx: np.ndarray             # (mg, nx+1, ny)
    qy: np.ndarray             # (mg, nx, ny+1)
    q0x: np.ndarray
    q0y: np.ndarray
    nonlin: list               # [N1, N2], each (mg, nx-1, ny-1)
    Fb: np.ndarray             # (nf,)
    CD: np.ndarray
    CL: np.ndarray

    def copy(self):
        return IBState(self.Gamma.copy(), self.psi.copy(), self.qx.copy(), self.qy.copy(),
                       self.q0x.copy(), self.q0y.copy(), [n.copy() for n in self.nonlin],
                       self.Fb.copy(), self.CD.copy(), self.CL.copy())


def linearize(prob, base_state):
    """LinearizedIBProblem(base_state, base_prob, dt) (problem-types.jl:65-86):
    the same model and matrices, with ΓB = base Γ and QB = avg_flux of the
    base state INCLUDING its base flux (the IBProblem avg_flux,
    problem-types.jl:78-83).  Returns a shallow copy of ``prob``."""
    import copy
    lp = copy.copy(prob)
    QBx, QBy = avg_flux(base_state.qx, base_state.qy, base_state.q0x, base_state.q0y, prob.grid)
    lp.base = (base_state.Gamma.copy(), QBx, QBy)
    return lp


def base_flux(prob, t=0.0):
    """timestepping.jl:252-270 (InertialMotion): uniform q0 per level; zero
    for a linearized problem (timestepping.jl:236-250); for a MovingGrid
    (:273-318) solid-body rotation plus translation,
    q0x = YY·(−hc Ω) + hc Ux0 and q0y = XX·(hc Ω) + hc Uy0 on each level."""
    g = prob.grid
    if prob.base is not None:
        return np.zeros((g.mg, g.nx + 1, g.ny)), np.zeros((g.mg, g.nx, g.ny + 1))
    if isinstance(prob.motion, MovingGrid):
        Om, Ux0, Uy0 = moving_grid_rates(prob, t)
        q0x = np.zeros((g.mg, g.nx + 1, g.ny))
        q0y = np.zeros((g.mg, g.nx, g.ny + 1))
        for lev in range(g.mg):
            hc = g.hc(lev)
            q0x[lev] = prob.YY[lev][None, :] * ((-hc) * Om) + hc * Ux0
            q0y[lev] = prob.XX[lev][:, None] * (hc * Om) + hc * Uy0
        return q0x, q0y
    a = prob.inclination
    q0x = np.zeros((g.mg, g.nx + 1, g.ny))
    q0y = np.zeros((g.mg, g.nx, g.ny + 1))
    for lev in range(g.mg):
        hc = g.hc(lev)
        q0x[lev] = (prob.Ux * math.cos(a) - prob.Uy * math.sin(a)) * hc
        q0y[lev] = (prob.Ux * math.sin(a) + prob.Uy * math.cos(a)) * hc
    return q0x, q0y


def make_state(prob):
    """IBState(prob), state-types.jl:25-47."""
    g = prob.grid
    sh = (g.mg, g.nx - 1, g.ny - 1)
    q0x, q0y = base_flux(prob, 0.0)
    return IBState(Gamma=np.zeros(sh), psi=np.zeros(sh),
                   qx=np.zeros((g.mg, g.nx + 1, g.ny)), qy=np.zeros((g.mg, g.nx, g.ny + 1)),
                   q0x=q0x, q0y=q0y, nonlin=[np.zeros(sh), np.zeros(sh)],
                   Fb=np.zeros(prob.nf), CD=np.zeros(len(prob.bodies)), CL=np.zeros(len(prob.bodies)))


def refresh_flux(state, prob):
    """vort2flux!(state.ψ, state.q, state.Γ, …) — makes ψ and q consistent
    with Γ (also coarsifies Γ into the coarse-level centres)."""
    state.psi, state.qx, state.qy = vort2flux(state.Gamma, prob.Lam, prob.grid)


def get_trial_state(state, prob):
    """timestepping.jl:86-129.  Returns (Γs, ψ, qsx, qsy) and updates
    state.nonlin (both slots equal afterwards)."""
    g = prob.grid
    dt = prob.dt
    Gs = np.zeros_like(state.Gamma)
    N1 = np.zeros_like(state.Gamma)
    for lev in range(g.mg - 1, -1, -1):
        hc = g.hc(lev)
        bc = np.zeros(g.nbc)
        rhsbc = np.zeros((g.nx - 1, g.ny - 1))
        if lev < g.mg - 1:
            bc = get_bc(state.Gamma[lev + 1], g)
            fac = 0.25 * dt / (prob.Re * hc ** 2)
            apply_bc(rhsbc, bc, fac, g)
        bc = bc * 0.25                                        # nonlinear.jl:183
        if prob.base is None:
            N1[lev] = nonlinear(state.Gamma[lev], state.qx[lev], state.qy[lev],
                                state.q0x[lev], state.q0y[lev], bc, hc, g)
        else:                                                 # nonlinear.jl:45-65,144-163
            GB, QBx, QBy = prob.base
            N1[lev] = nonlinear_linearized(state.Gamma[lev], state.qx[lev], state.qy[lev],
                                           GB[lev], QBx[lev], QBy[lev], bc, hc, g)
        state.nonlin[0][lev] = N1[lev]
        rhs = a_level(state.Gamma[lev], prob, lev)            # :111
        for n, b in enumerate(prob.beta):                     # :113-115
            rhs += (b * dt) * state.nonlin[n][lev]
        rhs += rhsbc                                          # :118
        Gs[lev] = ainv_level(rhs, prob, lev)                  # :121
    state.nonlin[1][...] = state.nonlin[0]                    # :125
    psi, qsx, qsy = vort2flux(Gs, prob.Lam, g)                # :127
    state.psi = psi
    return Gs, qsx, qsy


def update_stress(state, prob):
    """timestepping.jl:330-354."""
    g = prob.grid
    nb = prob.nb
    F = state.Fb.reshape((2, nb)).T                   # reshape(F̃b, nb, 2)
    t0 = 0
    for j, body in enumerate(prob.bodies):
        n = body.xb.shape[0]
        ds = body.ds
        fb = F[t0:t0 + n] * (g.h / prob.dt) / np.stack([ds, ds], axis=1)
        state.CD[j] = 2 * np.sum(ds * fb[:, 0])
        state.CL[j] = 2 * np.sum(ds * fb[:, 1])
        t0 += n


def advance(state, prob, t=0.0):
    """advance!(state, prob, t) for a Static body or a MovingGrid,
    timestepping.jl:35-67."""
    g = prob.grid
    if prob.moving_bodies:                                               # :39
        prob.move_bodies(t)
    if isinstance(prob.motion, MovingGrid):                              # :41-43
        state.q0x, state.q0y = base_flux(prob, t)
    Gs, qsx, qsy = get_trial_state(state, prob)                          # :52
    F = E_apply(qsx[0] + state.q0x[0], qsy[0] + state.q0y[0], prob)      # :154-159
    if prob.moving_bodies:                                               # :174-186: E(qs + q0) − ub·h
        F = F - np.concatenate([prob.ub[:, 0], prob.ub[:, 1]]) * g.h
    state.Fb = prob.Binv @ F                                             # :160
    update_stress(state, prob)                                           # :57
    state.Gamma = Gs.copy()                                              # :216
    src = ECt(state.Fb, prob)                                            # :217
    state.Gamma[0] -= ainv_level(src, prob, 0)                           # :218-220
    refresh_flux(state, prob)                                            # :64
    return state


def run(prob, state, nsteps, dt=None, record=True, t0=0.0):
    """Advance ``nsteps`` steps at t = t0 + k dt; returns (CD, CL) histories
    (nsteps, nbodies)."""
    cd = np.zeros((nsteps, len(prob.bodies)))
    cl = np.zeros((nsteps, len(prob.bodies)))
    for k in range(nsteps):
        advance(state, prob, t0 + k * prob.dt)
        cd[k] = state.CD
        cl[k] = state.CL
    return cd, cl
