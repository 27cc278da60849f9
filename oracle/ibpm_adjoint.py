"""Discrete adjoint of the static-body IBPM step (FP64, numpy).

THIS MODULE IS TEST INFRASTRUCTURE (the oracle), like ``ibpm_ref``: only
``tests/`` and the CPU legs of ``bench.py`` may import it, as the checker.

The reference (NUFgroup/IBPM.jl) has no adjoint; it has the forward step
``advance!`` (src/timestepping/timestepping.jl:35-67), restated in
``ibpm_ref.advance``, and a linearised problem (problem-types.jl:47-87).  This
module is the exact transpose of the derivative of ``ibpm_ref.advance``, one
operator at a time, so that gradients of functionals of a trajectory (for
example the time-averaged drag) can be checked against central finite
differences of ``ibpm_ref.run`` and used as the oracle of the GPU adjoint.

One step maps X_n = (Γ_n, q_n, N_{n-1}) to X_{n+1} (with q_n = curl ψ_n the
flux that vort2flux! made from Γ_n):

  1. per level: bc = get_bc!(Γ_n[l+1]); N_n = C'·DP(avg(q_n + q0), Γ_n, ¼bc)/(4hc²);
     rhs = A Γ_n + dt(β1 N_n + β2 N_{n-1}) + apply_bc!(0, bc, fac); Γs = A⁻¹ rhs
  2. Γs ← coarsify(Γs); qs = curl ψs (level 1)                  (vort2flux!)
  3. F̃ = B⁻¹ E(qs + q0)                                          (boundary_forces!)
  4. Γ' = Γs − e₁ A⁻¹₁ C'E' F̃                                     (project_circ!)
  5. Γ_{n+1} = coarsify(Γ'); q_{n+1} = curl ψ_{n+1}; N_n kept      (vort2flux!)

Everything but the product in the nonlinear term is linear with fixed
coefficients, so the adjoint of a step needs only (Γ_n, q_n).

Body-point positions xb enter through E (steps 3 and 4) and through
B = E M E' (M: C'-source on level 1 → A⁻¹₁ → vort2flux! → level-1 flux,
laplacian.jl:143-169).  With F̄ = B⁻ᵀ F̃̄ and r̄ = A⁻¹ Γ̄s (both formed by the
adjoint step anyway) the position gradient of a step is
  ∂J/∂xb += F̄ · ∂E/∂xb [q_{n+1,1} + q0]  −  F̃_n · ∂E/∂xb [C r̄₁]
because q_{n+1,1} = qs − M E'F̃ (so E(qs + q0) − B F̃ = E(q_{n+1,1} + q0)),
and C A⁻¹ Γ̄s₁ = C W + Mᵀ E' F̄ collects the E' and B terms of step 4.  The spectral
solves S diag(1/M) S·scale are symmetric (S, the 2-D DST-I matrix, is), and
so is the stencil A; B⁻¹ is not (B is not symmetric), so its transpose is
applied.  E' is the transpose of E (the same weights).
"""
from __future__ import annotations

import math

import numpy as np

from oracle import ibpm_ref as R


# --------------------------------------------------------------------------
# Transposes of the grid operators
# --------------------------------------------------------------------------
def get_bc_T(bbar, g):
    """Transpose of get_bc (mg-utils.jl:7-32): edge-vector adjoint → adjoint
    of the coarse field it was sampled from."""
    nx, ny = g.nx, g.ny
    B, T, L, Rt = g.BOT, g.TOP, g.LEFT, g.RIGHT
    r = np.zeros(bbar.shape[:-1] + (nx - 1, ny - 1))
    jb, jt = ny // 4 - 1, 3 * ny // 4 - 1
    il, ir = nx // 4 - 1, 3 * nx // 4 - 1
    i = nx // 4 + np.arange(0, nx // 2 + 1)
    ibc = np.arange(1, nx + 2, 2)
    r[..., i - 1, jb] += bbar[..., B + ibc - 1]
    r[..., i - 1, jt] += bbar[..., T + ibc - 1]
    i = nx // 4 + np.arange(1, nx // 2 + 1)
    ibc = np.arange(2, nx + 1, 2)
    r[..., i - 1, jb] += 0.5 * bbar[..., B + ibc - 1]
    r[..., i - 2, jb] += 0.5 * bbar[..., B + ibc - 1]
    r[..., i - 1, jt] += 0.5 * bbar[..., T + ibc - 1]
    r[..., i - 2, jt] += 0.5 * bbar[..., T + ibc - 1]
    j = ny // 4 + np.arange(0, ny // 2 + 1)
    jbc = np.arange(1, ny + 2, 2)
    r[..., il, j - 1] += bbar[..., L + jbc - 1]
    r[..., ir, j - 1] += bbar[..., Rt + jbc - 1]
    j = ny // 4 + np.arange(1, ny // 2 + 1)
    jbc = np.arange(2, ny + 1, 2)
    r[..., il, j - 1] += 0.5 * bbar[..., L + jbc - 1]
    r[..., il, j - 2] += 0.5 * bbar[..., L + jbc - 1]
    r[..., ir, j - 1] += 0.5 * bbar[..., Rt + jbc - 1]
    r[..., ir, j - 2] += 0.5 * bbar[..., Rt + jbc - 1]
    return r


def apply_bc_T(rbar, fac, g):
    """Transpose of apply_bc (mg-utils.jl:43-60) with respect to the edge
    vector: r̄ → fac · (edge rows and columns of r̄)."""
    nx, ny = g.nx, g.ny
    B, T, L, Rt = g.BOT, g.TOP, g.LEFT, g.RIGHT
    b = np.zeros(rbar.shape[:-2] + (g.nbc,))
    b[..., B + 1:B + nx] += fac * rbar[..., :, 0]
    b[..., T + 1:T + nx] += fac * rbar[..., :, ny - 2]
    b[..., L + 1:L + ny] += fac * rbar[..., 0, :]
    b[..., Rt + 1:Rt + ny] += fac * rbar[..., nx - 2, :]
    return b


def coarsify_T(Gbar, g, mg=None):
    """Transpose of the coarsify chain of vort2flux! (curl.jl:141-143,
    mg-utils.jl:71-106), in place on Gbar (..., mg, nx-1, ny-1): the centre of
    level l was overwritten by the restriction of level l-1, so its adjoint
    moves to level l-1 and the centre's own adjoint is cleared (coarsest
    level first, the reverse of the forward order)."""
    nx, ny = g.nx, g.ny
    mg = g.mg if mg is None else mg
    cx = slice(nx // 4, 3 * nx // 4 - 1)
    cy = slice(ny // 4, 3 * ny // 4 - 1)
    for lev in range(mg - 1, 0, -1):
        C = Gbar[..., lev, cx, cy].copy()
        Gbar[..., lev, cx, cy] = 0.0
        F = Gbar[..., lev - 1, :, :]
        F[..., 1:nx - 2:2, 1:ny - 2:2] += C
        for sx, sy in ((slice(2, nx - 1, 2), slice(1, ny - 2, 2)), (slice(1, nx - 2, 2), slice(2, ny - 1, 2)),
                       (slice(0, nx - 3, 2), slice(1, ny - 2, 2)), (slice(1, nx - 2, 2), slice(0, ny - 3, 2))):
            F[..., sx, sy] += 0.5 * C
        for sx, sy in ((slice(2, nx - 1, 2), slice(2, ny - 1, 2)), (slice(2, nx - 1, 2), slice(0, ny - 3, 2)),
                       (slice(0, nx - 3, 2), slice(0, ny - 3, 2)), (slice(0, nx - 3, 2), slice(2, ny - 1, 2))):
            F[..., sx, sy] += 0.25 * C
    return Gbar


def rot_T(Gbar, g):
    """Transpose of rot (C', curl.jl:22-34): Γ̄ → (q̄x, q̄y)."""
    nx, ny = g.nx, g.ny
    lead = Gbar.shape[:-2]
    qx = np.zeros(lead + (nx + 1, ny))
    qy = np.zeros(lead + (nx, ny + 1))
    qx[..., 1:nx, 0:ny - 1] += Gbar
    qx[..., 1:nx, 1:ny] -= Gbar
    qy[..., 1:nx, 1:ny] += Gbar
    qy[..., 0:nx - 1, 1:ny] -= Gbar
    return qx, qy


def curl_mg_T(qxb, qyb, g):
    """Transpose of curl_mg (curl.jl:81-116, with its bottom-row reading of
    ψbc[(B-1)+i]): (q̄x, q̄y) → (ψ̄, ψ̄bc)."""
    nx, ny = g.nx, g.ny
    B, T, L, Rt = g.BOT, g.TOP, g.LEFT, g.RIGHT
    lead = qxb.shape[:-2]
    p = np.zeros(lead + (nx - 1, ny - 1))
    b = np.zeros(lead + (g.nbc,))
    v = qxb[..., 1:nx, 1:ny - 1]
    p[..., :, 1:ny - 1] += v
    p[..., :, 0:ny - 2] -= v
    v = qxb[..., 1:nx, 0]
    p[..., :, 0] += v
    b[..., B:B + nx - 1] -= v
    v = qxb[..., 1:nx, ny - 1]
    b[..., T + 1:T + nx] += v
    p[..., :, ny - 2] -= v
    v = qxb[..., 0, :]
    b[..., L + 1:L + ny + 1] += v
    b[..., L:L + ny] -= v
    v = qxb[..., nx, :]
    b[..., Rt + 1:Rt + ny + 1] += v
    b[..., Rt:Rt + ny] -= v
    v = qyb[..., 1:nx - 1, 1:ny]
    p[..., 0:nx - 2, :] += v
    p[..., 1:nx - 1, :] -= v
    v = qyb[..., 0, 1:ny]
    b[..., L + 1:L + ny] += v
    p[..., 0, :] -= v
    v = qyb[..., nx - 1, 1:ny]
    p[..., nx - 2, :] += v
    b[..., Rt + 1:Rt + ny] -= v
    v = qyb[..., :, 0]
    b[..., B:B + nx] += v
    b[..., B + 1:B + nx + 1] -= v
    v = qyb[..., :, ny]
    b[..., T:T + nx] += v
    b[..., T + 1:T + nx + 1] -= v
    return p, b


def solves_T(qxb, qyb, Lam, g, mg=None):
    """Transpose of the level chain of vort2flux! after its coarsify chain
    (curl.jl:147-162): flux adjoints of every level (..., mg, ·, ·) → adjoint
    of the (coarsified) Γ.  Finest level first, the reverse of the forward."""
    mg = g.mg if mg is None else mg
    lead = qxb.shape[:-3]
    psib = np.zeros(lead + (mg, g.nx - 1, g.ny - 1))
    Gb = np.zeros_like(psib)
    scale = R.lap_inv_scale(g)
    for lev in range(mg):
        p, b = curl_mg_T(qxb[..., lev, :, :], qyb[..., lev, :, :], g)
        psib[..., lev, :, :] += p
        w = R.dst_inv(psib[..., lev, :, :], Lam, scale)       # Δ⁻¹ is symmetric
        Gb[..., lev, :, :] += w
        if lev < mg - 1:                                     # ψbc of the coarsest level is 0
            b = b + apply_bc_T(w, 1.0, g)
            psib[..., lev + 1, :, :] += get_bc_T(b, g)
    return Gb


def vort2flux_T(qxb, qyb, Lam, g, mg=None):
    """Transpose of vort2flux! (coarsify chain, then the level chain) with
    respect to its input Γ, for the flux outputs."""
    Gb = solves_T(qxb, qyb, Lam, g, mg)
    return coarsify_T(Gb, g, mg)


def nonlinear_T(Nb, G, qx, qy, q0x, q0y, Gbc, hc, g):
    """Transpose of the derivative of nonlinear (nonlinear.jl:168-201) at
    (G, q, q0, Gbc = ¼·bc): N̄ → (Ḡ, Ḡbc, q̄x, q̄y, Σq̄0x, Σq̄0y)."""
    nx, ny = g.nx, g.ny
    B, T, L, Rt = g.BOT, g.TOP, g.LEFT, g.RIGHT
    Qx, Qy = R.avg_flux(qx, qy, q0x, q0y, g)
    fxb, fyb = rot_T(Nb * (1.0 / (4 * hc ** 2)), g)
    Qxb = np.zeros_like(Qx)
    Qyb = np.zeros_like(Qy)
    Gb = np.zeros_like(G)
    bcb = np.zeros(g.nbc)
    # fqx rows (direct_product, nonlinear.jl:92-100)
    v = fxb[1:nx, 1:ny - 1]
    Qyb[1:nx, 2:ny] += v * G[:, 1:ny - 1]
    Gb[:, 1:ny - 1] += v * Qy[1:nx, 2:ny]
    Qyb[1:nx, 1:ny - 1] += v * G[:, 0:ny - 2]
    Gb[:, 0:ny - 2] += v * Qy[1:nx, 1:ny - 1]
    v = fxb[1:nx, 0]
    Qyb[1:nx, 1] += v * G[:, 0]
    Gb[:, 0] += v * Qy[1:nx, 1]
    Qyb[1:nx, 0] += v * Gbc[B + 1:B + nx]
    bcb[B + 1:B + nx] += v * Qy[1:nx, 0]
    v = fxb[1:nx, ny - 1]
    Qyb[1:nx, ny - 1] += v * G[:, ny - 2]
    Gb[:, ny - 2] += v * Qy[1:nx, ny - 1]
    Qyb[1:nx, ny] += v * Gbc[T + 1:T + nx]
    bcb[T + 1:T + nx] += v * Qy[1:nx, ny]
    # fqy columns (nonlinear.jl:102-110), scale -1
    v = -fyb[1:nx - 1, 1:ny]
    Qxb[2:nx, 1:ny] += v * G[1:nx - 1, :]
    Gb[1:nx - 1, :] += v * Qx[2:nx, 1:ny]
    Qxb[1:nx - 1, 1:ny] += v * G[0:nx - 2, :]
    Gb[0:nx - 2, :] += v * Qx[1:nx - 1, 1:ny]
    v = -fyb[0, 1:ny]
    Qxb[1, 1:ny] += v * G[0, :]
    Gb[0, :] += v * Qx[1, 1:ny]
    Qxb[0, 1:ny] += v * Gbc[L + 1:L + ny]
    bcb[L + 1:L + ny] += v * Qx[0, 1:ny]
    v = -fyb[nx - 1, 1:ny]
    Qxb[nx - 1, 1:ny] += v * G[nx - 2, :]
    Gb[nx - 2, :] += v * Qx[nx - 1, 1:ny]
    Qxb[nx, 1:ny] += v * Gbc[Rt + 1:Rt + ny]
    bcb[Rt + 1:Rt + ny] += v * Qx[nx, 1:ny]
    # avg_flux (nonlinear.jl:17-38)
    qxb = np.zeros_like(qx)
    qyb = np.zeros_like(qy)
    qxb[:, 1:ny] += Qxb[:, 1:ny]
    qxb[:, 0:ny - 1] += Qxb[:, 1:ny]
    qyb[1:nx, :] += Qyb[1:nx, :]
    qyb[0:nx - 1, :] += Qyb[1:nx, :]
    return Gb, bcb, qxb, qyb, 2.0 * Qxb[:, 1:ny].sum(), 2.0 * Qyb[1:nx, :].sum()


# --------------------------------------------------------------------------
# Objective and the adjoint of one step
# --------------------------------------------------------------------------
def cd_weights(prob):
    """∂(Σ_bodies CD)/∂F̃b: CD_j = 2 (h/dt) Σ F̃x over body j
    (update_stress!, timestepping.jl:330-354)."""
    w = np.zeros(prob.nf)
    w[:prob.nb] = 2.0 * prob.grid.h / prob.dt
    return w


def adjoint_step(prob, Gn, qxn, qyn, q0x, q0y, Gb1, qxb1, qyb1, Nb1, Fbar, xb_terms=None):
    """Adjoint of one ``ibpm_ref.advance`` from the state (Gn, qn) at the start
    of the step.  Inputs: the adjoints of the next state (Γ̄, q̄, N̄) and the
    direct sensitivity F̄ of the objective to this step's F̃b.  Returns the
    adjoints of this step's state and the per-level sums Σq̄0x, Σq̄0y; with
    ``xb_terms`` = (F̃_n, qx_{n+1} level 1, qy_{n+1} level 1) also this step's
    contribution to ∂J/∂xb, shape (nb, 2)."""
    g = prob.grid
    mg = g.mg
    dt = prob.dt
    q0xb = np.zeros(mg)
    q0yb = np.zeros(mg)
    # 5: Γ_{n+1} = coarsify(Γ'), q_{n+1} = curl ψ(Γ_{n+1})
    Gt = Gb1 + solves_T(qxb1, qyb1, prob.Lam, g)
    coarsify_T(Gt, g)
    # 4: Γ' = Γs − e₁ A⁻¹₁ C'E' F̃
    W = R.ainv_level(Gt[0], prob, 0)
    wx, wy = rot_T(W, g)
    Ft = Fbar - R.E_apply(wx, wy, prob)
    # 3: F̃ = B⁻¹ E(qs + q0)
    Fb_ = prob.Binv.T @ Ft
    qsx, qsy = R.flux_unflat(prob.ET @ Fb_, g)
    q0xb[0] += qsx.sum()
    q0yb[0] += qsy.sum()
    # 2: Γs ← coarsify(Γs); qs = curl ψs on level 1
    qxb = np.zeros((mg, g.nx + 1, g.ny))
    qyb = np.zeros((mg, g.nx, g.ny + 1))
    qxb[0], qyb[0] = qsx, qsy
    Gsb = Gt + solves_T(qxb, qyb, prob.Lam, g)
    coarsify_T(Gsb, g)
    # 1: the trial solve of every level
    rb = np.stack([R.ainv_level(Gsb[l], prob, l) for l in range(mg)])
    gxb = None
    if xb_terms is not None:
        Fn, qx1, qy1 = xb_terms
        cx, cy = rot_T(rb[0], g)
        gxb = R.dE_T(prob, Fb_, qx1 + q0x[0], qy1 + q0y[0]) - R.dE_T(prob, Fn, cx, cy)
    Gb = np.zeros_like(Gn)
    qxo = np.zeros_like(qxn)
    qyo = np.zeros_like(qyn)
    Nbo = prob.beta[1] * dt * rb
    Nbar = Nb1 + prob.beta[0] * dt * rb
    for lev in range(mg):
        hc = g.hc(lev)
        Gb[lev] += R.a_level(rb[lev], prob, lev)
        bcs = np.zeros(g.nbc)
        if lev < mg - 1:
            bcs = 0.25 * R.get_bc(Gn[lev + 1], g)
        gb, bcb, qxl, qyl, sx, sy = nonlinear_T(Nbar[lev], Gn[lev], qxn[lev], qyn[lev], q0x[lev], q0y[lev],
                                                bcs, hc, g)
        Gb[lev] += gb
        qxo[lev] += qxl
        qyo[lev] += qyl
        q0xb[lev] += sx
        q0yb[lev] += sy
        if lev < mg - 1:
            fac = 0.25 * dt / (prob.Re * hc ** 2)
            Gb[lev + 1] += get_bc_T(0.25 * bcb + apply_bc_T(rb[lev], fac, g), g)
    if xb_terms is not None:
        return Gb, qxo, qyo, Nbo, q0xb, q0yb, gxb
    return Gb, qxo, qyo, Nbo, q0xb, q0yb


# --------------------------------------------------------------------------
# Gradient of the time-averaged drag with checkpointed recomputation
# --------------------------------------------------------------------------
def _snapshot(st):
    return st.Gamma.copy(), st.qx.copy(), st.qy.copy(), st.nonlin[0].copy()


def _restore(st, snap):
    st.Gamma[...] = snap[0]
    st.qx[...] = snap[1]
    st.qy[...] = snap[2]
    st.nonlin[0][...] = snap[3]
    st.nonlin[1][...] = snap[3]


def mean_drag_gradient(prob, state, nsteps, window, k=50):
    """J = (1/window) Σ_{n > nsteps-window} Σ_bodies CD_n over ``nsteps``
    steps of ``ibpm_ref.advance`` from ``state`` (left unchanged).  The
    adjoint sweep recomputes each segment of ``k`` steps from its checkpoint.

    Returns (J, Γ̄_0, q̄_0x, q̄_0y, Σq̄0x[lev], Σq̄0y[lev]): the gradient of J
    with respect to the initial Γ, q (the nonlinear history enters through
    N_{-1} = state.nonlin) and the uniform base flux of every level."""
    return mean_force_gradient(prob, state, nsteps, window, k)


def force_weights(prob, w_cd, w_cl):
    """∂(Σ_bodies w_cd CD + w_cl CL)/∂F̃b (update_stress!, timestepping.jl:330-354)."""
    w = np.zeros(prob.nf)
    w[:prob.nb] = w_cd * 2.0 * prob.grid.h / prob.dt
    w[prob.nb:] = w_cl * 2.0 * prob.grid.h / prob.dt
    return w


def mean_force_gradient(prob, state, nsteps, window, k=50, w_cd=1.0, w_cl=0.0, want_xb=False):
    """J = (1/window) Σ_{n > nsteps-window} Σ_bodies (w_cd CD_n + w_cl CL_n);
    as mean_drag_gradient, and with ``want_xb`` the gradient with respect to
    the body-point positions (nb, 2) appended to the result."""
    g = prob.grid
    st = state.copy()
    ckpt = {}
    J = 0.0
    w = force_weights(prob, w_cd, w_cl)
    n0 = nsteps - window
    for n in range(nsteps):
        if n % k == 0:
            ckpt[n] = _snapshot(st)
        R.advance(st, prob)
        if n >= n0:
            J += float(np.sum(w_cd * st.CD + w_cl * st.CL)) / window
    Gb = np.zeros_like(st.Gamma)
    qxb = np.zeros_like(st.qx)
    qyb = np.zeros_like(st.qy)
    Nb = np.zeros_like(st.Gamma)
    q0xb = np.zeros(g.mg)
    q0yb = np.zeros(g.mg)
    gxb = np.zeros((prob.nb, 2))
    for s in sorted(ckpt, reverse=True):
        e = min(s + k, nsteps)
        _restore(st, ckpt[s])
        tape = []
        for n in range(s, e):
            Gn, qxn, qyn = st.Gamma.copy(), st.qx.copy(), st.qy.copy()
            R.advance(st, prob)
            tape.append((Gn, qxn, qyn, st.Fb.copy(), st.qx[0].copy(), st.qy[0].copy()))
        for n in range(e - 1, s - 1, -1):
            Gn, qxn, qyn, Fn, qx1, qy1 = tape[n - s]
            Fbar = w / window if n >= n0 else np.zeros(prob.nf)
            out = adjoint_step(prob, Gn, qxn, qyn, st.q0x, st.q0y, Gb, qxb, qyb, Nb, Fbar,
                               xb_terms=(Fn, qx1, qy1) if want_xb else None)
            Gb, qxb, qyb, Nb, sx, sy = out[:6]
            if want_xb:
                gxb += out[6]
            q0xb += sx
            q0yb += sy
    if want_xb:
        return J, Gb, qxb, qyb, q0xb, q0yb, gxb
    return J, Gb, qxb, qyb, q0xb, q0yb


def initial_vorticity_gradient(prob, Gb0, qxb0, qyb0):
    """Chain the adjoint of the initial state through its construction from a
    finest-level vorticity ω: Γ₀ = coarsify([h²ω, 0, …]), q₀ = curl ψ(Γ₀)
    (vort2flux!).  Returns ∂J/∂ω (nx-1, ny-1)."""
    g = prob.grid
    Gt = Gb0 + solves_T(qxb0, qyb0, prob.Lam, g)
    coarsify_T(Gt, g)
    return g.h ** 2 * Gt[0]


def angle_gradient(prob, q0xb, q0yb):
    """∂J/∂α from the per-level base-flux sums: q0x = (Ux cos α − Uy sin α) hc,
    q0y = (Ux sin α + Uy cos α) hc (timestepping.jl:252-270)."""
    g = prob.grid
    a = prob.inclination
    d = 0.0
    for lev in range(g.mg):
        hc = g.hc(lev)
        d += q0xb[lev] * (-prob.Ux * math.sin(a) - prob.Uy * math.cos(a)) * hc
        d += q0yb[lev] * (prob.Ux * math.cos(a) - prob.Uy * math.sin(a)) * hc
    return d
