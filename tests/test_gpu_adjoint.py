"""Discrete adjoint on the GPU (ibpm_adjoint_run, through the C ABI) against
the oracle's adjoint (oracle/ibpm_adjoint.py, itself checked against finite
differences of the oracle's forward step) and against central differences
of the GPU forward run."""
import numpy as np
import pytest

from ibpm_cases import gpu_problem, oracle_problem, rel

pytestmark = pytest.mark.gpu
NSTEPS, WINDOW, K = 24, 8, 5


def _omega(prob_grid, seed=4):
    rng = np.random.default_rng(seed)
    return 1e-4 * rng.standard_normal((prob_grid.nx - 1, prob_grid.ny - 1))


def _gpu_start(gp, w):
    """Γ = h²ω on the finest level, zero history, then vort2flux! (the same
    construction as the oracle's)."""
    import ibpm_gpu as G
    st = G.IBState(gp)
    for a in (st.Gamma, st.q, st.psi, st.nonlin[0], st.nonlin[1], st.Fb):
        a[...] = 0.0
    st.Gamma[:, 0] = gp.grid.h ** 2 * w.flatten(order="F")
    G.push_state(st, gp)
    G.vort2flux(st, gp)
    return st


@pytest.mark.parametrize("name", ["sq64_mg3", "rect64x32_mg2_two"])
def test_adjoint_matches_oracle(name):
    import ibpm_gpu as G
    from oracle import ibpm_adjoint as A
    from oracle import ibpm_ref as R
    op = oracle_problem(name)
    gp = gpu_problem(name)
    w = _omega(op.grid)
    _gpu_start(gp, w)
    res = G.adjoint_run(gp, NSTEPS, K, WINDOW, w_cd=1.0, w_cl=0.5)
    st = R.make_state(op)
    st.Gamma[0] = op.grid.h ** 2 * w
    R.refresh_flux(st, op)
    # the oracle objective with the same weights: mean over the window of Σ(CD + ½ CL)
    J, Gb, qxb, qyb, q0xb, q0yb = _oracle_gradient(A, op, st, w_cd=1.0, w_cl=0.5)
    assert abs(res.J - J) <= 1e-11 * abs(J), name
    assert rel(res.grad_Gamma0, R.gamma_to_ref(Gb)) < 1e-9, name
    assert rel(res.grad_q0, R.flux_to_ref(qxb, qyb)) < 1e-9, name
    gw = A.initial_vorticity_gradient(op, Gb, qxb, qyb)
    assert rel(res.grad_omega0, gw.flatten(order="F")) < 1e-9, name
    ga = A.angle_gradient(op, q0xb, q0yb)
    assert abs(res.grad_alpha - ga) <= 1e-9 * max(abs(ga), np.max(np.abs(gw)) * 1e-3), name
    gp.close()


def _oracle_gradient(A, prob, state, w_cd, w_cl):
    """The oracle's gradient of the mean of Σ(w_cd CD + w_cl CL) over the window."""
    return A.mean_force_gradient(prob, state, NSTEPS, WINDOW, k=K, w_cd=w_cd, w_cl=w_cl)


def test_adjoint_matches_gpu_finite_differences():
    """⟨∂J/∂ω, d⟩ against (J(ω + εd) − J(ω − εd)) / 2ε through the GPU forward
    run, ε = 1e-6 on a unit-variance direction."""
    import ibpm_gpu as G
    gp = gpu_problem("sq64_mg3")
    w = _omega(gp.grid)
    d = np.random.default_rng(9).standard_normal(w.shape)
    _gpu_start(gp, w)
    res = G.adjoint_run(gp, NSTEPS, K, WINDOW)

    def J(wv):
        st = _gpu_start(gp, wv)
        cd, _ = G.advance(st, gp, 0.0, nsteps=NSTEPS)
        return float(np.mean(np.sum(cd[-WINDOW:], axis=1)))
    eps = 1e-6
    fd = (J(w + eps * d) - J(w - eps * d)) / (2 * eps)
    ad = float(np.dot(res.grad_omega0, d.flatten(order="F")))
    assert abs(fd - ad) <= 1e-5 * abs(fd)
    gp.close()


def test_adjoint_checkpoint_interval_and_final_state():
    """The recomputation reproduces the forward run exactly: the gradient does
    not depend on the checkpoint interval, and the handle ends at the state
    that ibpm_advance reaches."""
    import ibpm_gpu as G
    gp = gpu_problem("sq64_mg3")
    w = _omega(gp.grid)
    grads = []
    for k in (1, 7, NSTEPS):
        _gpu_start(gp, w)
        grads.append(G.adjoint_run(gp, NSTEPS, k, WINDOW))
    for r in grads[1:]:
        assert np.array_equal(r.grad_Gamma0, grads[0].grad_Gamma0)
        assert np.array_equal(r.grad_q0, grads[0].grad_q0)
        assert r.J == grads[0].J
    after_adj = G.IBState(gp)
    G.pull_state(after_adj, gp)
    st = _gpu_start(gp, w)
    G.advance(st, gp, 0.0, nsteps=NSTEPS)
    assert np.array_equal(after_adj.Gamma, st.Gamma) and np.array_equal(after_adj.q, st.q)
    gp.close()


def test_refined_adjoint_close_to_fp64():
    """The adjoint over an FP32-refined forward run gives the FP64 gradient to
    within the refined path's tolerance."""
    import ibpm_gpu as G
    out = []
    for prec in ("fp64", "fp32_refined"):
        gp = gpu_problem("sq64_mg3", precision=prec)
        _gpu_start(gp, _omega(gp.grid))
        out.append(G.adjoint_run(gp, NSTEPS, K, WINDOW))
        gp.close()
    assert abs(out[1].J - out[0].J) <= 1e-6 * abs(out[0].J)
    assert rel(out[1].grad_omega0, out[0].grad_omega0) < 1e-5


# Body-point positions.  Bodies are moved off the grid lines first: the
# reference's smoothed delta jumps by ~1e-9 at |r| = h, 2h, 3h, which finite
# differences would pick up where grid samples sit exactly at those distances.
OFF = np.array([0.01234, -0.00711])


def _pair_xb(name, seed):
    """Oracle and GPU problems of case ``name`` with the bodies moved by OFF,
    both started from the same seeded random state."""
    import ibpm_gpu as G
    from oracle import ibpm_ref as R
    from ibpm_cases import CASES, build_bodies, random_state, to_gpu_state
    c = CASES[name]
    og = R.make_grid(c["h"], c["bnd"], c["mg"])
    ob = build_bodies(R, c["bodies"], og.h)
    for b in ob:
        b.xb = b.xb + OFF
    Ux, Uy, a = c["fs"]
    op = R.IBProblem(grid=og, bodies=ob, dt=c["dt"], Re=c["Re"], Ux=Ux, Uy=Uy, inclination=a)
    ost = random_state(op, seed=seed)
    gp = _gpu_with_xb(name, np.concatenate([b.xb for b in ob]))
    gst = G.IBState(gp)
    to_gpu_state(ost, gst)
    G.push_state(gst, gp)
    return op, ost, gp, gst


def _gpu_with_xb(name, xb):
    import ibpm_gpu as G
    from ibpm_cases import CASES, build_bodies
    c = CASES[name]
    g = G.make_grid(c["h"], c["bnd"], c["mg"])
    bodies, t0 = build_bodies(G, c["bodies"], g.h), 0
    for b in bodies:
        n = b.xb.shape[0]
        b.xb = xb[t0:t0 + n].copy()
        t0 += n
    return G.IBProblem(g, bodies, c["dt"], c["Re"], freestream=c["fs"])


def test_position_gradient_matches_oracle():
    """∂J/∂xb of the mean total lift (two bodies, inclined free stream) against
    the oracle's position adjoint, itself checked by central differences."""
    import ibpm_gpu as G
    from oracle import ibpm_adjoint as A
    op, ost, gp, _ = _pair_xb("rect64x32_mg2_two", seed=9)
    res = G.adjoint_run(gp, 16, 4, 6, w_cd=0.3, w_cl=1.0, want_xb=True)
    J, *_, gxb = A.mean_force_gradient(op, ost, 16, 6, k=4, w_cd=0.3, w_cl=1.0, want_xb=True)
    assert abs(res.J - J) <= 1e-11 * abs(J)
    assert rel(res.grad_xb, gxb) < 1e-9
    # asking for it leaves the other gradients as they were
    op2, ost2, gp2, _ = _pair_xb("rect64x32_mg2_two", seed=9)
    res2 = G.adjoint_run(gp2, 16, 4, 6, w_cd=0.3, w_cl=1.0)
    assert np.array_equal(res2.grad_Gamma0, res.grad_Gamma0) and res2.grad_xb is None
    gp.close()
    gp2.close()


def test_position_gradient_matches_gpu_finite_differences():
    """The mean total lift over the last 10 of 30 steps, its gradient with
    respect to all body-point positions along 8 seeded unit-variance
    directions against central differences of the GPU forward run
    (E and B⁻¹ rebuilt on the device for each moved body), ε = 1e-5 h.  The
    bound scales with ‖∇J‖‖d‖: a direction nearly orthogonal to the gradient
    has a small projection whose finite difference is mostly round-off (the
    oracle's own differences show the same, 4e-6 of such a projection)."""
    import ibpm_gpu as G
    from ibpm_cases import to_gpu_state
    op, ost, gp, _ = _pair_xb("sq64_mg3", seed=12)
    nsteps, window = 30, 10
    res = G.adjoint_run(gp, nsteps, 10, window, w_cd=0.0, w_cl=1.0, want_xb=True)
    xb0 = op.xb.copy()
    eps = 1e-5 * op.grid.h

    def J(xb):
        p = _gpu_with_xb("sq64_mg3", xb)
        st = G.IBState(p)
        to_gpu_state(ost, st)
        G.push_state(st, p)
        _, cl = G.advance(st, p, 0.0, nsteps=nsteps)
        p.close()
        return float(np.mean(np.sum(cl[-window:], axis=1)))
    assert abs(J(xb0) - res.J) <= 1e-12 * abs(res.J)
    rng = np.random.default_rng(2024)
    for _ in range(8):
        d = rng.standard_normal(xb0.shape)
        fd = (J(xb0 + eps * d) - J(xb0 - eps * d)) / (2 * eps)
        ad = float(np.sum(res.grad_xb * d))
        assert abs(fd - ad) <= 1e-6 * np.linalg.norm(res.grad_xb) * np.linalg.norm(d), (fd, ad)
    gp.close()
