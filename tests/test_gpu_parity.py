"""FP64 GPU path (through the C ABI) against the FP64 oracle.  The bar is
1e-10 relative (max-norm error over max-norm of the oracle field)."""
import numpy as np
import pytest

from ibpm_cases import CASES, gpu_problem, oracle_problem, random_state, rel, to_gpu_state

pytestmark = pytest.mark.gpu
TOL = 1e-10
SMALL = ["sq64_mg3", "rect64x32_mg2_two", "sq64_mg1_plate"]


@pytest.fixture(scope="module", params=SMALL)
def pair(request):
    return request.param, oracle_problem(request.param), gpu_problem(request.param)


def test_binv(pair):
    name, op, gp = pair
    assert rel(gp.binv(), op.Binv) < 1e-8, name     # inverse of B: limited by cond(B)·ε


def test_vort2flux(pair):
    import ibpm_gpu as G
    from oracle import ibpm_ref as R
    name, op, gp = pair
    rng = np.random.default_rng(11)
    ost = R.make_state(op)
    ost.Gamma = rng.standard_normal(ost.Gamma.shape)
    gst = G.IBState(gp)
    gst.Gamma[:] = R.gamma_to_ref(ost.Gamma)
    G.push_state(gst, gp, fields=("Gamma",))
    G.vort2flux(gst, gp)
    R.refresh_flux(ost, op)
    assert rel(gst.Gamma, R.gamma_to_ref(ost.Gamma)) < 1e-14, name   # coarsify is a stencil
    assert rel(gst.psi, R.gamma_to_ref(ost.psi)) < TOL, name
    assert rel(gst.q, R.flux_to_ref(ost.qx, ost.qy)) < TOL, name


@pytest.mark.parametrize("nsteps", [1, 15])
def test_step_from_random_state(pair, nsteps):
    import ibpm_gpu as G
    from oracle import ibpm_ref as R
    name, op, gp = pair
    ost = random_state(op, seed=7 + nsteps)
    gst = G.IBState(gp)
    to_gpu_state(ost, gst)
    G.push_state(gst, gp)
    cd, cl = G.advance(gst, gp, 0.0, nsteps=nsteps)
    ocd, ocl = R.run(op, ost, nsteps)
    assert rel(gst.Gamma, R.gamma_to_ref(ost.Gamma)) < TOL, name
    assert rel(gst.psi, R.gamma_to_ref(ost.psi)) < TOL, name
    assert rel(gst.q, R.flux_to_ref(ost.qx, ost.qy)) < TOL, name
    assert rel(gst.nonlin[0], R.gamma_to_ref(ost.nonlin[0])) < TOL, name
    assert rel(gst.nonlin[1], R.gamma_to_ref(ost.nonlin[1])) < TOL, name
    assert rel(gst.Fb[:, 0], ost.Fb) < TOL, name
    assert rel(cd, ocd) < TOL and rel(cl, ocl) < TOL, name


def test_cyl200_mg3_500_steps():
    """The 200x200, 3-level, 157-point cylinder at Re=40 (h=0.02,
    dt=0.004) from rest for 500 steps: CD/CL histories and the final
    vorticity agree with the oracle to 1e-10."""
    import ibpm_gpu as G
    from oracle import ibpm_ref as R
    op = oracle_problem("cyl200_mg3")
    gp = gpu_problem("cyl200_mg3")
    ost = R.make_state(op)
    gst = G.IBState(gp)
    cd, cl = G.advance(gst, gp, 0.0, nsteps=500)
    ocd, ocl = R.run(op, ost, 500)
    assert rel(cd, ocd) < TOL
    # CL is round-off-sized for the symmetric flow: compare against max |CD|
    assert np.max(np.abs(cl - ocl)) / np.max(np.abs(ocd)) < TOL
    assert rel(gst.Gamma, R.gamma_to_ref(ost.Gamma)) < TOL
    assert rel(gst.q, R.flux_to_ref(ost.qx, ost.qy)) < TOL


def test_determinism():
    """Two handles on the same problem give bit-identical states."""
    import ibpm_gpu as G
    out = []
    for _ in range(2):
        gp = gpu_problem("sq64_mg3")
        gst = G.IBState(gp)
        cd, cl = G.advance(gst, gp, 0.0, nsteps=30)
        out.append((gst.Gamma.copy(), cd.copy()))
        gp.close()
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])
