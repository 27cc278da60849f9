"""Transform plans (ibpm_set_transform_plan, through the C ABI): the radix-8
throughput plan computes the same step as the radix-4 latency plan, to the
oracle's 1e-10 in FP64 and within the FP32-refined tolerances, for launches
over one level and over several, and a batch's tuned plan is the plan its
members' own handles reproduce bit for bit."""
import numpy as np
import pytest

from ibpm_cases import CASES, build_bodies, gpu_problem, oracle_problem, random_state, rel, to_gpu_state

pytestmark = pytest.mark.gpu
TOL = 1e-10
SMALL = ["sq64_mg3", "rect64x32_mg2_two", "sq64_mg1_plate"]
LAT, THR, AUTO = 0, 1, 2


def _run(gp, op, seed, nsteps):
    import ibpm_gpu as G
    from oracle import ibpm_ref as R
    ost = random_state(op, seed=seed)
    gst = G.IBState(gp)
    to_gpu_state(ost, gst)
    G.push_state(gst, gp)
    cd, cl = G.advance(gst, gp, 0.0, nsteps=nsteps)
    ocd, ocl = R.run(op, ost, nsteps)
    return gst, ost, cd, cl, ocd, ocl


@pytest.mark.parametrize("name", SMALL)
@pytest.mark.parametrize("plans", [(THR, THR), (LAT, THR), (THR, LAT)])
def test_fp64_plans_match_oracle(name, plans):
    import ibpm_gpu as G
    from oracle import ibpm_ref as R
    op = oracle_problem(name)
    gp = gpu_problem(name)
    G.set_transform_plan(gp, *plans)
    assert G.transform_plan(gp) == plans
    gst, ost, cd, cl, ocd, ocl = _run(gp, op, 17, 15)
    assert rel(gst.Gamma, R.gamma_to_ref(ost.Gamma)) < TOL, (name, plans)
    assert rel(gst.psi, R.gamma_to_ref(ost.psi)) < TOL, (name, plans)
    assert rel(gst.q, R.flux_to_ref(ost.qx, ost.qy)) < TOL, (name, plans)
    assert rel(gst.Fb[:, 0], ost.Fb) < TOL, (name, plans)
    assert rel(cd, ocd) < TOL and rel(cl, ocl) < TOL, (name, plans)
    gp.close()


@pytest.mark.parametrize("name", SMALL)
def test_refined_throughput_plan_matches_oracle(name):
    """Two sweeps: the FP64 result (1e-10); one sweep: within 1e-6.  CL is
    compared on the force scale (the larger of max |CD| and max |CL|): on
    sq64_mg3 |CL| stays below 0.53 against |CD| up to 413, and one sweep's
    FP32 error there was 1.2e-6 of max |CL| with this plan (4.8e-7 with the
    latency plan), 1.5e-9 of the force."""
    import ibpm_gpu as G
    from oracle import ibpm_ref as R
    op = oracle_problem(name)
    for sweeps, tol in ((2, 1e-10), (1, 1e-6)):
        gp = gpu_problem(name, precision="fp32_refined", refine_sweeps=sweeps)
        G.set_transform_plan(gp, THR, THR)
        gst, ost, cd, cl, ocd, ocl = _run(gp, op, 23, 15)
        scale = max(np.max(np.abs(ocd)), np.max(np.abs(ocl)))
        assert rel(gst.Gamma, R.gamma_to_ref(ost.Gamma)) < tol, (name, sweeps)
        assert rel(cd, ocd) < tol, (name, sweeps)
        assert np.max(np.abs(cl - ocl)) / scale < tol, (name, sweeps)
        gp.close()


def test_cyl200_throughput_plan_matches_oracle():
    """N = 200 (radices 8, 5, 5 against 4, 5, 5, 2): 500 steps from rest, as
    the latency plan's test.  (After 50 steps both plans are 1.25e-10 from
    the oracle in Γ, to four digits alike: the rounding of B⁻¹ on a vorticity
    that is still small, not the transforms.)"""
    import ibpm_gpu as G
    from oracle import ibpm_ref as R
    op = oracle_problem("cyl200_mg3")
    gp = gpu_problem("cyl200_mg3")
    G.set_transform_plan(gp, THR, THR)
    ost = R.make_state(op)
    gst = G.IBState(gp)
    cd, cl = G.advance(gst, gp, 0.0, nsteps=500)
    ocd, ocl = R.run(op, ost, 500)
    assert rel(cd, ocd) < TOL
    assert np.max(np.abs(cl - ocl)) / np.max(np.abs(ocd)) < TOL
    assert rel(gst.Gamma, R.gamma_to_ref(ost.Gamma)) < TOL
    gp.close()


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("fp32_refined", 1e-6)])
def test_plans_agree_at_512(precision, tol):
    """512² × 2 levels (beyond the oracle's quick sizes): both plans from the
    same vortex start agree within the parity bar in FP64 (the rounding of the
    two factorisations, amplified by the Schur solve) and within the refined
    tolerance in FP32-refined form."""
    import ibpm_gpu as G
    out = []
    for plans in ((LAT, LAT), (THR, THR)):
        g = G.make_grid(0.01, (-1.0, 4.12, -2.56, 2.56), 2)
        p = G.IBProblem(g, [G.make_cylinder(0.5, g.h, 0.0, 0.0, n=314)], 0.002, 100.0,
                        freestream=(1.0, 0.0, 0.0), precision=precision, sync_fields=False)
        G.set_transform_plan(p, *plans)
        st = G.IBState(p)
        x = (np.arange(1, g.nx) * g.h - g.offx)[:, None]
        y = (np.arange(1, g.ny) * g.h - g.offy)[None, :]
        w = 1e-3 * np.exp(-((x - 1.5) ** 2 + (y - 0.1) ** 2) / 0.04)
        st.Gamma[:, 0] = (g.h * g.h * w).reshape(-1, order="F")
        G.push_state(st, p, fields=("Gamma",))
        G.vort2flux(st, p)
        cd, cl = G.advance(st, p, 0.0, nsteps=5)
        G.pull_state(st, p)
        out.append((cd, cl, np.array(st.Gamma)))
        p.close()
    (cd0, cl0, g0), (cd1, cl1, g1) = out
    assert rel(cd1, cd0) < tol
    assert np.max(np.abs(cl1 - cl0)) / np.max(np.abs(cd0)) < tol
    assert rel(g1, g0) < tol


def test_plan_arguments_are_checked():
    import ibpm_gpu as G
    gp = gpu_problem("sq64_mg1_plate")
    assert G.transform_plan(gp) == (LAT, AUTO)
    with pytest.raises(G.IBPMError):
        G.set_transform_plan(gp, AUTO, LAT)            # AUTO is for multi-slab launches only
    with pytest.raises(G.IBPMError):
        G.set_transform_plan(gp, LAT, -1)
    assert G.transform_plan(gp) == (LAT, AUTO)
    G.set_transform_plan(gp, THR, LAT)
    assert G.transform_plan(gp) == (THR, LAT)
    gp.close()


def _spec(name, prec):
    import ibpm_gpu as G
    c = CASES[name]
    g = G.make_grid(c["h"], c["bnd"], c["mg"])
    return dict(grid=g, bodies=build_bodies(G, c["bodies"], g.h), dt=c["dt"], Re=c["Re"], freestream=c["fs"],
                precision=prec)


@pytest.mark.parametrize("plan", [LAT, THR])
def test_batch_plan_is_the_members_plan(plan):
    """A batch with its members' single-level launches on `plan` computes
    exactly what each member's problem computes alone on that plan."""
    import ibpm_gpu as G
    members = [("sq64_mg3", "fp64"), ("sq64_mg1_plate", "fp32_refined"), ("rect64x32_mg2_two", "fp64")]
    specs = [_spec(n, p) for n, p in members]
    batch = G.Batch(specs, lanes=2)
    batch.set_plan(plan)
    assert batch.plan == plan
    starts = []
    for i, (name, _) in enumerate(members):
        ost = random_state(oracle_problem(name), seed=50 + i)
        st = G.IBState(batch.members[i])
        to_gpu_state(ost, st)
        G.push_state(st, batch.members[i])
        starts.append(ost)
    forces = batch.advance(12)
    for i, (name, prec) in enumerate(members):
        sp = specs[i]
        solo = G.IBProblem(sp["grid"], sp["bodies"], sp["dt"], sp["Re"], freestream=sp["freestream"],
                           precision=prec, sync_fields=False)
        G.set_transform_plan(solo, plan, AUTO)
        st = G.IBState(solo)
        to_gpu_state(starts[i], st)
        G.push_state(st, solo)
        cd, cl = G.advance(st, solo, 0.0, nsteps=12)
        assert np.array_equal(forces[i][0], cd) and np.array_equal(forces[i][1], cl), (name, prec, plan)
        solo.close()
    batch.close()


def test_batch_member_plan_change_is_refused():
    """A member's plan belongs to its batch: changed on the member's own
    handle, the next batch step is refused instead of running stale graphs."""
    import ibpm_gpu as G
    batch = G.Batch([_spec("sq64_mg3", "fp64"), _spec("sq64_mg1_plate", "fp64")], lanes=2)
    batch.advance(1)
    G.set_transform_plan(batch.members[0], THR, LAT)
    with pytest.raises(G.IBPMError):
        batch.advance(1)
    batch.close()
