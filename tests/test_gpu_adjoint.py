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
    """mean_drag_gradient generalised to the weights (w_cd, w_cl): the force
    weights of the objective enter only through the step's F̃b sensitivity."""
    saved = A.cd_weights

    def weights(p):
        w = np.zeros(p.nf)
        w[:p.nb] = w_cd * 2.0 * p.grid.h / p.dt
        w[p.nb:] = w_cl * 2.0 * p.grid.h / p.dt
        return w
    A.cd_weights = weights
    try:
        out = A.mean_drag_gradient(prob, state, NSTEPS, WINDOW, k=K)
    finally:
        A.cd_weights = saved
    # J from the oracle run itself (mean_drag_gradient sums CD only)
    st = state.copy()
    cd, cl = __import__("oracle.ibpm_ref", fromlist=["run"]).run(prob, st, NSTEPS)
    J = float(np.mean(np.sum(w_cd * cd[-WINDOW:] + w_cl * cl[-WINDOW:], axis=1)))
    return (J,) + out[1:]


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
