"""Failures the host can see, made on the host (no GPU fault): a non-finite
state, a null or closed handle, a bad step count or field shape.  The
reference stops its run loop on a non-finite lift coefficient
(src/ibpm.jl:95-97); the library reports IBPM_ERR_NONFINITE with the force
history up to that step, and the handle stays usable."""
import ctypes

import numpy as np
import pytest

from ibpm_cases import gpu_problem, oracle_problem, random_state, rel, to_gpu_state

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp64", "fp32_refined"])
def test_nan_in_state_reports_nonfinite(precision):
    import ibpm_gpu as G
    from oracle import ibpm_ref as R
    op = oracle_problem("sq64_mg3")
    gp = gpu_problem("sq64_mg3", precision=precision)
    st = G.IBState(gp)
    to_gpu_state(random_state(op, seed=3), st)
    st.Gamma[100, 0] = np.nan
    G.push_state(st, gp)
    with pytest.raises(G.IBPMError) as e:
        G.advance(st, gp, 0.0, nsteps=4)
    assert e.value.code == G.IBPM_ERR_NONFINITE
    assert e.value.CL.shape == (4, 1) and not np.all(np.isfinite(e.value.CL))
    assert not np.all(np.isfinite(st.CL))          # as the reference leaves state.CL
    # run_sim stops at the first non-finite lift, as run_sim! does
    G.push_state(st, gp)
    cd, cl = G.run_sim(np.arange(6) * gp.dt, st, gp)
    assert cl.shape[0] >= 1 and not np.all(np.isfinite(cl[-1]))
    assert np.all(np.isfinite(cl[:-1]))
    # the handle recovers from a finite state: the run matches the oracle
    ost = random_state(op, seed=4)
    to_gpu_state(ost, st)
    G.push_state(st, gp)
    cd, _ = G.advance(st, gp, 0.0, nsteps=3)
    ocd, _ = R.run(op, ost, 3)
    assert rel(cd, ocd) < (1e-10 if precision == "fp64" else 1e-6)
    gp.close()


def test_null_and_closed_handles():
    import ibpm_gpu as G
    lib = G.load_library()
    assert lib.ibpm_advance(None, 0.0, 1, None, None) == G.IBPM_ERR_INVALID
    assert lib.ibpm_sync(None) == G.IBPM_ERR_INVALID
    gp = gpu_problem("sq64_mg3")
    st = G.IBState(gp)
    gp.close()
    with pytest.raises(G.IBPMError) as e:
        G.advance(st, gp, 0.0, nsteps=1)
    assert e.value.code == G.IBPM_ERR_INVALID


def test_bad_step_count_and_shapes():
    import ibpm_gpu as G
    gp = gpu_problem("sq64_mg3")
    st = G.IBState(gp)
    assert gp.lib.ibpm_advance(gp.handle, 0.0, -1, None, None) == G.IBPM_ERR_INVALID
    cd, cl = G.advance(st, gp, 0.0, nsteps=0)
    assert cd.shape == (0, 1)
    st.Gamma = np.zeros((st.Gamma.shape[0] - 1, st.Gamma.shape[1]))
    with pytest.raises(G.IBPMError) as e:
        G.push_state(st, gp)
    assert e.value.code == G.IBPM_ERR_INVALID and "shape" in str(e.value)
    with pytest.raises(G.IBPMError):
        G.pull_state(st, gp)
    gp.close()
