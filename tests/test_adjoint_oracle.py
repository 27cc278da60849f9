"""The oracle's discrete adjoint (oracle/ibpm_adjoint.py) against the forward
oracle: dot-product identities for every transposed operator, the adjoint of
one step against central differences (a step is quadratic in its state, so
central differences are exact up to round-off), and the checkpointed
gradient of the time-averaged drag against central finite differences."""
import numpy as np
import pytest

from ibpm_cases import oracle_problem, random_state

from oracle import ibpm_adjoint as A
from oracle import ibpm_ref as R


@pytest.fixture(scope="module")
def prob():
    return oracle_problem("sq64_mg3")


def _dot(*pairs):
    return sum(float(np.sum(a * b)) for a, b in pairs)


def test_operator_transposes(prob):
    g = prob.grid
    rng = np.random.default_rng(1)
    sh = (g.nx - 1, g.ny - 1)
    x, y = rng.standard_normal(sh), rng.standard_normal(g.nbc)
    assert np.isclose(_dot((R.get_bc(x, g), y)), _dot((x, A.get_bc_T(y, g))), rtol=1e-13)
    r = np.zeros(sh)
    R.apply_bc(r, y, 0.7, g)
    z = rng.standard_normal(sh)
    assert np.isclose(_dot((r, z)), _dot((y, A.apply_bc_T(z, 0.7, g))), rtol=1e-13)
    qx, qy = rng.standard_normal((g.nx + 1, g.ny)), rng.standard_normal((g.nx, g.ny + 1))
    bx, by = A.rot_T(z, g)
    assert np.isclose(_dot((R.rot(qx, qy, g), z)), _dot((qx, bx), (qy, by)), rtol=1e-13)
    cx, cy = R.curl_mg(x, y, g)
    p, b = A.curl_mg_T(qx, qy, g)
    assert np.isclose(_dot((cx, qx), (cy, qy)), _dot((x, p), (y, b)), rtol=1e-13)
    G = rng.standard_normal((g.mg,) + sh)
    Gc = G.copy()
    for lev in range(1, g.mg):
        R.coarsify(Gc[lev], Gc[lev - 1], g)
    H = rng.standard_normal(G.shape)
    assert np.isclose(_dot((Gc, H)), _dot((G, A.coarsify_T(H.copy(), g))), rtol=1e-13)
    qxb = rng.standard_normal((g.mg, g.nx + 1, g.ny))
    qyb = rng.standard_normal((g.mg, g.nx, g.ny + 1))
    _, fx, fy = R.vort2flux(G.copy(), prob.Lam, g)
    assert np.isclose(_dot((fx, qxb), (fy, qyb)), _dot((G, A.vort2flux_T(qxb, qyb, prob.Lam, g))), rtol=1e-12)


def test_nonlinear_transpose(prob):
    """The bilinear nonlinear term: ⟨N̄, dN⟩ from a central difference equals
    the adjoint pairing with (dΓ, dΓbc, dq, dq0)."""
    g = prob.grid
    rng = np.random.default_rng(2)
    G = rng.standard_normal((g.nx - 1, g.ny - 1))
    bc = rng.standard_normal(g.nbc)
    qx, qy = rng.standard_normal((g.nx + 1, g.ny)), rng.standard_normal((g.nx, g.ny + 1))
    q0x, q0y = np.full(qx.shape, 0.3), np.full(qy.shape, -0.2)
    dG, dbc = rng.standard_normal(G.shape), rng.standard_normal(bc.shape)
    dqx, dqy = rng.standard_normal(qx.shape), rng.standard_normal(qy.shape)
    d0x, d0y = 0.4, -0.9
    Nb = rng.standard_normal(G.shape)
    hc = 0.5
    eps = 1e-3

    def N(s):
        return R.nonlinear(G + s * dG, qx + s * dqx, qy + s * dqy, q0x + s * d0x, q0y + s * d0y, bc + s * dbc, hc, g)
    fd = _dot((Nb, (N(eps) - N(-eps)) / (2 * eps)))
    gb, bcb, qxb, qyb, sx, sy = A.nonlinear_T(Nb, G, qx, qy, q0x, q0y, bc, hc, g)
    ad = _dot((gb, dG), (bcb, dbc), (qxb, dqx), (qyb, dqy)) + sx * d0x + sy * d0y
    assert abs(fd - ad) <= 1e-10 * abs(fd)


def test_step_adjoint_matches_central_differences(prob):
    g = prob.grid
    rng = np.random.default_rng(3)
    st = random_state(prob, seed=5)
    Gb1 = rng.standard_normal(st.Gamma.shape)
    qxb1, qyb1 = rng.standard_normal(st.qx.shape), rng.standard_normal(st.qy.shape)
    Nb1 = rng.standard_normal(st.Gamma.shape)
    Fbar = rng.standard_normal(prob.nf)
    d = dict(G=1e-3 * rng.standard_normal(st.Gamma.shape), qx=1e-3 * rng.standard_normal(st.qx.shape),
             qy=1e-3 * rng.standard_normal(st.qy.shape), N=1e-3 * rng.standard_normal(st.Gamma.shape))

    def phi(s):
        x = st.copy()
        x.Gamma = x.Gamma + s * d["G"]
        x.qx = x.qx + s * d["qx"]
        x.qy = x.qy + s * d["qy"]
        x.nonlin = [x.nonlin[0] + s * d["N"], x.nonlin[1] + s * d["N"]]
        R.advance(x, prob)
        return _dot((Gb1, x.Gamma), (qxb1, x.qx), (qyb1, x.qy), (Nb1, x.nonlin[1]), (Fbar, x.Fb))
    fd = (phi(1.0) - phi(-1.0)) / 2.0
    Gb, qxb, qyb, Nb, _, _ = A.adjoint_step(prob, st.Gamma, st.qx, st.qy, st.q0x, st.q0y, Gb1, qxb1, qyb1, Nb1, Fbar)
    ad = _dot((Gb, d["G"]), (qxb, d["qx"]), (qyb, d["qy"]), (Nb, d["N"]))
    assert abs(fd - ad) <= 1e-9 * abs(fd)


def test_mean_drag_gradient_matches_finite_differences(prob):
    """∂J/∂ω₀ along a random unit-variance direction and ∂J/∂α, J the mean
    drag over the last 8 of 24 steps from a seeded N(0, 1e-4) vorticity
    perturbation, checkpoint every 5 steps; central differences, ε = 1e-6."""
    g = prob.grid
    rng = np.random.default_rng(4)
    w0 = 1e-4 * rng.standard_normal((g.nx - 1, g.ny - 1))
    dirn = rng.standard_normal(w0.shape)
    nsteps, window = 24, 8

    def state_from(w, alpha):
        p = prob if alpha == prob.inclination else _with_angle(prob, alpha)
        st = R.make_state(p)
        st.Gamma[0] = g.h ** 2 * w
        R.refresh_flux(st, p)
        return p, st

    p, st = state_from(w0, prob.inclination)
    J, Gb, qxb, qyb, q0xb, q0yb = A.mean_drag_gradient(p, st, nsteps, window, k=5)
    gw = A.initial_vorticity_gradient(p, Gb, qxb, qyb)

    def J_of(w, alpha):
        pp, s = state_from(w, alpha)
        cd, _ = R.run(pp, s, nsteps)
        return float(np.mean(np.sum(cd[-window:], axis=1)))
    eps = 1e-6
    fd_w = (J_of(w0 + eps * dirn, 0.0) - J_of(w0 - eps * dirn, 0.0)) / (2 * eps)
    assert abs(J - J_of(w0, 0.0)) <= 1e-13 * abs(J)
    print("dJ/dw: fd %.12e adjoint %.12e" % (fd_w, float(np.sum(gw * dirn))))
    assert abs(fd_w - float(np.sum(gw * dirn))) <= 1e-5 * abs(fd_w)
    # the mean drag is even in α at α = 0 (a zero derivative); check at α = 0.1
    a0 = 0.1
    p1, st1 = state_from(w0, a0)
    _, Gb, qxb, qyb, q0xb, q0yb = A.mean_drag_gradient(p1, st1, nsteps, window, k=5)
    ga = A.angle_gradient(p1, q0xb, q0yb)
    fd_a = (J_of(w0, a0 + eps) - J_of(w0, a0 - eps)) / (2 * eps)
    assert abs(fd_a - ga) <= 1e-5 * abs(fd_a)


def _with_angle(prob, alpha):
    """The same problem with freestream angle α (B and E do not depend on it)."""
    import copy
    p = copy.copy(prob)
    p.inclination = alpha
    return p


# Finite differences in xb: the reference's δh (rounded coefficients) jumps by
# up to ~3e-9 at |r| = h, 2h, 3h, and a body point on a grid line puts grid
# samples exactly there, so the bodies are first moved off the grid lines.
OFF = np.array([0.01234, -0.00711])


def _with_xb(prob, xb):
    """The same problem with body points moved to ``xb`` (E and B rebuilt)."""
    bodies, t0 = [], 0
    for b in prob.bodies:
        n = b.xb.shape[0]
        bodies.append(R.Body(xb=xb[t0:t0 + n].copy(), ds=b.ds.copy()))
        t0 += n
    return R.IBProblem(grid=prob.grid, bodies=bodies, dt=prob.dt, Re=prob.Re, Ux=prob.Ux, Uy=prob.Uy,
                       inclination=prob.inclination)


def test_delta_derivative_matches_central_differences():
    h = 0.0625
    rb = 0.0313
    rf = rb + h * np.linspace(-3.2, 3.2, 4001)
    eps = 1e-7
    fd = (R.delta_h(rf, rb + eps, h) - R.delta_h(rf, rb - eps, h)) / (2 * eps)
    an = R.delta_h_db(rf, rb, h)
    r1 = np.abs(rf - rb) / h
    away = np.abs(r1 - np.round(r1)) > 1e-4      # the rounded coefficients leave ~1e-9 jumps at r = h, 2h, 3h
    assert np.max(np.abs(fd - an)[away]) <= 1e-7 * np.max(np.abs(an))


def test_step_position_adjoint_matches_central_differences(prob):
    """One step: the xb part of the step adjoint against central differences of
    ⟨adjoint weights, step outputs⟩ with E and B rebuilt at moved points."""
    prob = _with_xb(prob, prob.xb + OFF)
    rng = np.random.default_rng(13)
    st = random_state(prob, seed=8)
    Gb1 = rng.standard_normal(st.Gamma.shape)
    qxb1, qyb1 = rng.standard_normal(st.qx.shape), rng.standard_normal(st.qy.shape)
    Nb1 = rng.standard_normal(st.Gamma.shape)
    Fbar = rng.standard_normal(prob.nf)
    dx = rng.standard_normal(prob.xb.shape)
    eps = 1e-6 * prob.grid.h

    def phi(s):
        p = _with_xb(prob, prob.xb + s * dx)
        x = st.copy()
        R.advance(x, p)
        return _dot((Gb1, x.Gamma), (qxb1, x.qx), (qyb1, x.qy), (Nb1, x.nonlin[1]), (Fbar, x.Fb))
    fd = (phi(eps) - phi(-eps)) / (2 * eps)
    x = st.copy()
    R.advance(x, prob)
    out = A.adjoint_step(prob, st.Gamma, st.qx, st.qy, st.q0x, st.q0y, Gb1, qxb1, qyb1, Nb1, Fbar,
                         xb_terms=(x.Fb, x.qx[0], x.qy[0]))
    ad = float(np.sum(out[6] * dx))
    print("step d/dxb: fd %.12e adjoint %.12e" % (fd, ad))
    assert abs(fd - ad) <= 1e-6 * abs(fd)


def test_mean_lift_position_gradient_matches_finite_differences():
    """∂J/∂xb of the mean total lift over the last 6 of 16 steps (two bodies,
    an inclined free stream, seeded state; checkpoint every 4 steps) along a
    random direction of all body points, against central differences with E
    and B rebuilt at the moved points."""
    prob2 = oracle_problem("rect64x32_mg2_two")
    prob2 = _with_xb(prob2, prob2.xb + OFF)
    rng = np.random.default_rng(21)
    st = random_state(prob2, seed=9)
    nsteps, window = 16, 6
    J, *_, gxb = A.mean_force_gradient(prob2, st, nsteps, window, k=4, w_cd=0.0, w_cl=1.0, want_xb=True)
    dx = rng.standard_normal(prob2.xb.shape)
    eps = 1e-6 * prob2.grid.h

    def J_of(s):
        p = _with_xb(prob2, prob2.xb + s * dx)
        _, cl = R.run(p, st.copy(), nsteps)
        return float(np.mean(np.sum(cl[-window:], axis=1)))
    assert abs(J - J_of(0.0)) <= 1e-12 * abs(J)
    fd = (J_of(eps) - J_of(-eps)) / (2 * eps)
    ad = float(np.sum(gxb * dx))
    print("dJ/dxb: fd %.12e adjoint %.12e" % (fd, ad))
    assert abs(fd - ad) <= 1e-5 * abs(fd)
