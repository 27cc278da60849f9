"""The large two-body workload: two cylinders (D = 1, 628 points each, centres
(0, ±0.75)) at Re = 150 on 1024x1024 cells x 5 levels, h = 0.005, dt = 0.001
(src/timestepping/timestepping.jl:35-67 on the geometry of
examples/double_cyl.jl:19-28).  Its Schur complement (nf = 2512) is inverted by
the blocked Gauss–Jordan elimination.  The cylinders are moved off the grid
lines by ~1e-7 (ibpm_cases.OFF_GRID): points on grid lines sample δh on its
rounded-coefficient jumps, where a one-ulp move of a point moves the results
by ~1e-9.

The oracle's own B at this size takes tens of minutes on the host, so B⁻¹ is
checked column-wise instead: the oracle's B_times! (laplacian.jl:143-169) of a
few unit vectors, multiplied by the device's B⁻¹, gives the unit vectors to
the accuracy an inverse has, 10·n·ε·cond₂(B), with ‖B⁻¹‖₂ from the device's
inverse and ‖B‖₂ by power iteration on the oracle's B.  The steps are then
checked against the oracle run with the device's B⁻¹ (every other operator
the oracle's own): FP64 to 1e-10, FP32-refined to 1e-6 (CL on the force
scale)."""
import numpy as np
import pytest

import bench
from ibpm_cases import rel, to_gpu_state

pytestmark = pytest.mark.gpu
C5 = dict(h=0.005, mg=5, Re=150.0, dt=0.001, nb=628, centres=(0.75, -0.75))


def _centres():
    from ibpm_cases import OFF_GRID
    return [(OFF_GRID[0], y + OFF_GRID[1]) for y in C5["centres"]]


def _oracle(build_binv=False):
    from oracle import ibpm_ref as R
    g = R.make_grid(C5["h"], bench.BOUNDARY, C5["mg"])
    bodies = [R.make_cylinder(0.5, g.h, x, y, n=C5["nb"]) for x, y in _centres()]
    return R.IBProblem(grid=g, bodies=bodies, dt=C5["dt"], Re=C5["Re"], build_binv=build_binv)


def _gpu(precision="fp64"):
    import ibpm_gpu as G
    g = G.make_grid(C5["h"], bench.BOUNDARY, C5["mg"])
    bodies = [G.make_cylinder(0.5, g.h, x, y, n=C5["nb"]) for x, y in _centres()]
    return G.IBProblem(g, bodies, C5["dt"], C5["Re"], freestream=(1.0, 0.0, 0.0), precision=precision)


@pytest.fixture(scope="module")
def pair():
    op = _oracle()
    gp = _gpu()
    op.Binv = gp.binv()
    yield op, gp
    gp.close()


def test_grid_and_bodies(pair):
    op, gp = pair
    assert (op.grid.nx, op.grid.ny, op.nf) == (1024, 1024, 2512)


def test_binv_inverts_the_oracles_B(pair):
    from oracle import ibpm_ref as R
    op, gp = pair
    cols = [0, 627, 1300, 2511]
    Z = np.zeros((op.nf, len(cols)))
    Z[cols, np.arange(len(cols))] = 1.0
    Bc = R.B_times(op, Z)
    X = op.Binv @ Bc
    E = np.zeros_like(X)
    for j, c in enumerate(cols):
        E[c, j] = 1.0
    # ‖B‖₂ by power iteration (B is symmetric to 1e-5)
    z = np.random.default_rng(4).standard_normal((op.nf, 1))
    for _ in range(4):
        z = R.B_times(op, z / np.linalg.norm(z))
    normB = float(np.linalg.norm(z))
    normBinv = np.linalg.norm(op.Binv, 2)
    bound = 10.0 * op.nf * np.finfo(float).eps * normB * normBinv
    assert np.max(np.abs(X - E)) < bound, (float(np.max(np.abs(X - E))), float(bound), float(normB * normBinv))


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("fp32_refined", 1e-6)])
def test_steps_match_oracle(pair, precision, tol):
    import ibpm_gpu as G
    from ibpm_cases import random_state
    from oracle import ibpm_ref as R
    from ibpm_cases import force_scale_err
    op, gp64 = pair
    gp = gp64 if precision == "fp64" else _gpu(precision)
    ost = random_state(op, seed=17, amp=1e-4)
    st = G.IBState(gp)
    to_gpu_state(ost, st)
    G.push_state(st, gp)
    cd, cl = G.advance(st, gp, 0.0, nsteps=3)
    G.pull_state(st, gp)
    if gp is not gp64:
        gp.close()
    ocd, ocl = R.run(op, ost, 3)
    assert rel(cd, ocd) < tol and force_scale_err(cl, ocl, ocd) < tol
    assert rel(st.Gamma, R.gamma_to_ref(ost.Gamma)) < tol
    assert rel(st.q, R.flux_to_ref(ost.qx, ost.qy)) < tol
