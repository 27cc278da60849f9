"""Level chains of vort2flux! (ibpm_set_level_chain, through the C ABI): the
reference's sequential order (src/fluid-operators/curl.jl:133-165) and the
boundary transfer compute the same step, to the oracle's 1e-10 in FP64 and
within the FP32-refined tolerance, also when the chain is changed between
steps of one run; a batch's chain is the one its members' own handles
reproduce bit for bit."""
import numpy as np
import pytest

from ibpm_cases import CASES, build_bodies, force_scale_err, gpu_problem, oracle_problem, random_state, rel, \
    to_gpu_state

pytestmark = pytest.mark.gpu
SEQ, BT = 0, 1
CASES_MG = ["sq64_mg3", "rect64x32_mg2_two"]


def _start(gp, op, seed):
    import ibpm_gpu as G
    ost = random_state(op, seed=seed)
    gst = G.IBState(gp)
    to_gpu_state(ost, gst)
    G.push_state(gst, gp)
    return gst, ost


@pytest.mark.parametrize("name", CASES_MG)
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("fp32_refined", 1e-6)])
def test_sequential_chain_matches_oracle(name, precision, tol):
    import ibpm_gpu as G
    from oracle import ibpm_ref as R
    op = oracle_problem(name)
    gp = gpu_problem(name, precision=precision)
    assert G.level_chain(gp) == BT
    G.set_level_chain(gp, SEQ)
    assert G.level_chain(gp) == SEQ
    gst, ost = _start(gp, op, 41)
    cd, cl = G.advance(gst, gp, 0.0, nsteps=12)
    G.pull_state(gst, gp)
    ocd, ocl = R.run(op, ost, 12)
    assert rel(cd, ocd) < tol and force_scale_err(cl, ocl, ocd) < tol, name
    assert rel(gst.Gamma, R.gamma_to_ref(ost.Gamma)) < tol, name
    assert rel(gst.q, R.flux_to_ref(ost.qx, ost.qy)) < tol, name
    gp.close()


def test_sequential_chain_cyl200_from_rest():
    """The 200x200, 3-level cylinder from rest for 300 steps with the
    sequential chain: CD/CL and the final vorticity within 1e-10 of the
    oracle (from a random start of amplitude 1e-3 the small vorticity leaves
    B⁻¹'s rounding at 3.6e-10 of it, for either chain)."""
    import ibpm_gpu as G
    from oracle import ibpm_ref as R
    op = oracle_problem("cyl200_mg3")
    gp = gpu_problem("cyl200_mg3")
    G.set_level_chain(gp, SEQ)
    ost = R.make_state(op)
    gst = G.IBState(gp)
    cd, cl = G.advance(gst, gp, 0.0, nsteps=300)
    G.pull_state(gst, gp)
    ocd, ocl = R.run(op, ost, 300)
    assert rel(cd, ocd) < 1e-10 and force_scale_err(cl, ocl, ocd) < 1e-10
    assert rel(gst.Gamma, R.gamma_to_ref(ost.Gamma)) < 1e-10
    gp.close()


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("fp32_refined", 1e-6)])
def test_chain_change_between_steps(precision, tol):
    """Steps with the boundary transfer, then the sequential chain, then the
    boundary transfer again, in one run (the step graphs are captured again
    at each change): the history matches the oracle's run."""
    import ibpm_gpu as G
    from oracle import ibpm_ref as R
    name = "sq64_mg3"
    op = oracle_problem(name)
    gp = gpu_problem(name, precision=precision)
    gst, ost = _start(gp, op, 43)
    cds, cls = [], []
    t = 0.0
    for chain in (BT, SEQ, BT):
        G.set_level_chain(gp, chain)
        cd, cl = G.advance(gst, gp, t, nsteps=5)
        cds.append(cd)
        cls.append(cl)
        t += 5 * gp.dt
    G.pull_state(gst, gp)
    ocd, ocl = R.run(op, ost, 15)
    cd, cl = np.concatenate(cds), np.concatenate(cls)
    assert rel(cd, ocd) < tol and force_scale_err(cl, ocl, ocd) < tol
    assert rel(gst.Gamma, R.gamma_to_ref(ost.Gamma)) < tol
    gp.close()


def test_chain_arguments_are_checked():
    import ibpm_gpu as G
    gp = gpu_problem("sq64_mg3")
    with pytest.raises(G.IBPMError) as e:
        G.set_level_chain(gp, 7)
    assert e.value.code == G.IBPM_ERR_INVALID
    assert G.level_chain(gp) == BT
    gp.close()
    # one level has no chain: either setting is kept and the step is the same
    gp1 = gpu_problem("sq64_mg1_plate")
    for chain in (SEQ, BT):
        G.set_level_chain(gp1, chain)
        assert G.level_chain(gp1) == chain
    gp1.close()


def _spec(name, prec):
    import ibpm_gpu as G
    c = CASES[name]
    g = G.make_grid(c["h"], c["bnd"], c["mg"])
    return dict(grid=g, bodies=build_bodies(G, c["bodies"], g.h), dt=c["dt"], Re=c["Re"], freestream=c["fs"],
                precision=prec)


@pytest.mark.parametrize("chain", [SEQ, BT])
def test_batch_chain_is_the_members_chain(chain):
    import ibpm_gpu as G
    members = [("sq64_mg3", "fp64"), ("sq64_mg3", "fp32_refined"), ("rect64x32_mg2_two", "fp64")]
    specs = [_spec(n, p) for n, p in members]
    batch = G.Batch(specs, lanes=2)
    batch.set_chain(chain)
    assert batch.chain == chain
    for i, (name, _) in enumerate(members):
        _start(batch.members[i], oracle_problem(name), 50 + i)
    forces = batch.advance(10)
    for i, (name, prec) in enumerate(members):
        sp = specs[i]
        solo = G.IBProblem(sp["grid"], sp["bodies"], sp["dt"], sp["Re"], freestream=sp["freestream"],
                           precision=prec, sync_fields=False)
        G.set_transform_plan(solo, batch.plan, G.IBPM_PLAN_AUTO)
        G.set_level_chain(solo, chain)
        st, _ = _start(solo, oracle_problem(name), 50 + i)
        cd, cl = G.advance(st, solo, 0.0, nsteps=10)
        assert np.array_equal(forces[i][0], cd) and np.array_equal(forces[i][1], cl), (name, prec)
        solo.close()
    # a member's chain changed on its own is refused
    G.set_level_chain(batch.members[0], 1 - chain)
    with pytest.raises(G.IBPMError):
        batch.advance(1)
    batch.close()
