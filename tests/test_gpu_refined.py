"""FP32-refined path (through the C ABI) against the FP64 oracle.

The mode runs the sine transforms of every Poisson-type solve in FP32 and
corrects each solve with FP64-residual refinement sweeps started from the
previous solution.  With two sweeps the result is the FP64 result (1e-10);
with one sweep (the default) each solve keeps the FP32 error of one
correction, relative to the change of its solution per step, and the forces
stay within 1e-6 of the oracle."""
import numpy as np
import pytest

from ibpm_cases import gpu_problem, oracle_problem, random_state, rel, to_gpu_state

pytestmark = pytest.mark.gpu
SMALL = ["sq64_mg3", "rect64x32_mg2_two", "sq64_mg1_plate"]


@pytest.mark.parametrize("name", SMALL)
@pytest.mark.parametrize("sweeps,tol_state,tol_force", [(2, 1e-10, 1e-10), (1, 1e-6, 1e-6)])
def test_refined_steps_from_random_state(name, sweeps, tol_state, tol_force):
    import ibpm_gpu as G
    from oracle import ibpm_ref as R
    op = oracle_problem(name)
    gp = gpu_problem(name, precision="fp32_refined", refine_sweeps=sweeps)
    for nsteps in (1, 15):
        ost = random_state(op, seed=7 + nsteps)
        gst = G.IBState(gp)
        to_gpu_state(ost, gst)
        G.push_state(gst, gp)
        cd, cl = G.advance(gst, gp, 0.0, nsteps=nsteps)
        ocd, ocl = R.run(op, ost, nsteps)
        for fld, ref in ((gst.Gamma, R.gamma_to_ref(ost.Gamma)), (gst.psi, R.gamma_to_ref(ost.psi)),
                         (gst.q, R.flux_to_ref(ost.qx, ost.qy)), (gst.nonlin[0], R.gamma_to_ref(ost.nonlin[0]))):
            assert rel(fld, ref) < tol_state, (name, nsteps)
        assert rel(cd, ocd) < tol_force and rel(cl, ocl) < tol_force, (name, nsteps)
    gp.close()


def test_refined_cyl200_mg3_500_steps():
    """The 200x200, 3-level, 157-point cylinder at Re=40 from rest, 500 steps
    with one sweep: CD within 1e-6 (relative), CL within 1e-6 of max |CD|
    (the flow is symmetric: CL is round-off sized), vorticity within 1e-6
    (relative L2)."""
    import ibpm_gpu as G
    from oracle import ibpm_ref as R
    op = oracle_problem("cyl200_mg3")
    gp = gpu_problem("cyl200_mg3", precision="fp32_refined")
    ost = R.make_state(op)
    gst = G.IBState(gp)
    cd, cl = G.advance(gst, gp, 0.0, nsteps=500)
    ocd, ocl = R.run(op, ost, 500)
    assert np.max(np.abs(cd - ocd) / np.abs(ocd)) < 1e-6
    assert np.max(np.abs(cl - ocl)) / np.max(np.abs(ocd)) < 1e-6
    og = R.gamma_to_ref(ost.Gamma)
    assert np.linalg.norm(gst.Gamma - og) / np.linalg.norm(og) < 1e-6
    gp.close()


def test_refined_rejects_bad_sweeps():
    import ibpm_gpu as G
    with pytest.raises(G.IBPMError):
        gpu_problem("sq64_mg3", precision="fp32_refined", refine_sweeps=99)
