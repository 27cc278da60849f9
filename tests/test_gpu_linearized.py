"""The linearised problem (ibpm_set_base_state: LinearizedIBProblem of
problem-types.jl:47-87) on the GPU against the oracle's, through the C ABI:
every field and CD/CL to 1e-10 after 1 and 15 steps, on nested grids (where
the reference's edge-value quirk matters) and on a single grid."""
import numpy as np
import pytest

from ibpm_cases import gpu_problem, oracle_problem, random_state, rel, to_gpu_state

pytestmark = pytest.mark.gpu
TOL = 1e-10


@pytest.mark.parametrize("name", ["sq64_mg3", "rect64x32_mg2_two", "sq64_mg1_plate"])
@pytest.mark.parametrize("nsteps", [1, 15])
def test_linearized_step_matches_oracle(name, nsteps):
    import ibpm_gpu as G
    from oracle import ibpm_ref as R
    op = oracle_problem(name)
    gp = gpu_problem(name)
    base = random_state(op, seed=40)
    gbase = G.IBState(gp)
    to_gpu_state(base, gbase)
    gp.set_base_state(gbase)
    lp = R.linearize(op, base)
    ost = random_state(op, seed=41 + nsteps, amp=1e-4)
    ost.q0x[...] = 0.0
    ost.q0y[...] = 0.0
    gst = G.IBState(gp)
    assert not np.any(gst.q0)                   # the perturbation carries no base flux
    to_gpu_state(ost, gst)
    G.push_state(gst, gp)
    cd, cl = G.advance(gst, gp, 0.0, nsteps=nsteps)
    ocd, ocl = R.run(lp, ost, nsteps)
    assert rel(gst.Gamma, R.gamma_to_ref(ost.Gamma)) < TOL, name
    assert rel(gst.q, R.flux_to_ref(ost.qx, ost.qy)) < TOL, name
    assert rel(gst.nonlin[0], R.gamma_to_ref(ost.nonlin[0])) < TOL, name
    assert rel(cd, ocd) < TOL and rel(cl, ocl) < TOL, name
    gp.close()


def test_adjoint_refuses_linearized_handle():
    import ibpm_gpu as G
    gp = gpu_problem("sq64_mg3")
    gp.set_base_state(G.IBState(gp))
    with pytest.raises(G.IBPMError) as e:
        G.adjoint_run(gp, 4, 2, 2)
    assert e.value.code == G.IBPM_ERR_UNSUPPORTED
    gp.close()
