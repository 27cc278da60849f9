"""Batches of independent simulations (ibpm_batch_*, through the C ABI): a
member of a batch computes exactly what the same problem computes on its own
handle — the batch only runs the members' steps side by side."""
import numpy as np
import pytest

from ibpm_cases import CASES, build_bodies, oracle_problem, random_state, to_gpu_state

pytestmark = pytest.mark.gpu
MEMBERS = [("sq64_mg3", "fp64"), ("rect64x32_mg2_two", "fp64"), ("sq64_mg1_plate", "fp32_refined"),
           ("sq64_mg3", "fp32_refined")]
NSTEPS = 20


def _spec(name, prec):
    import ibpm_gpu as G
    c = CASES[name]
    g = G.make_grid(c["h"], c["bnd"], c["mg"])
    return dict(grid=g, bodies=build_bodies(G, c["bodies"], g.h), dt=c["dt"], Re=c["Re"], freestream=c["fs"],
                precision=prec)


def _start(m, name, seed):
    import ibpm_gpu as G
    ost = random_state(oracle_problem(name), seed=seed)
    st = G.IBState(m)
    to_gpu_state(ost, st)
    G.push_state(st, m)


@pytest.mark.parametrize("lanes", [0, 1])
def test_batch_members_match_single_runs(lanes):
    import ibpm_gpu as G
    specs = [_spec(n, p) for n, p in MEMBERS]
    batch = G.Batch(specs, lanes=lanes)
    assert 1 <= batch.lanes <= len(MEMBERS)
    for i, (name, _) in enumerate(MEMBERS):
        _start(batch.members[i], name, seed=30 + i)
    forces = batch.advance(NSTEPS)
    for i, (name, prec) in enumerate(MEMBERS):
        sp = specs[i]
        solo = G.IBProblem(sp["grid"], sp["bodies"], sp["dt"], sp["Re"], freestream=sp["freestream"],
                           precision=prec, sync_fields=False)
        # the tuner also chooses the members' transform plan for single-level
        # launches and their level chain (per group of one grid)
        G.set_transform_plan(solo, *G.transform_plan(batch.members[i]))
        G.set_level_chain(solo, G.level_chain(batch.members[i]))
        _start(solo, name, seed=30 + i)
        st = G.IBState(solo)
        cd, cl = G.advance(st, solo, 0.0, nsteps=NSTEPS)
        G.pull_state(st, solo)
        bst = G.IBState(batch.members[i])
        assert np.array_equal(forces[i][0], cd) and np.array_equal(forces[i][1], cl), (name, prec)
        assert np.array_equal(bst.Gamma, st.Gamma) and np.array_equal(bst.q, st.q), (name, prec)
        solo.close()
    batch.close()


def test_batch_rejects_members_stepped_alone():
    import ibpm_gpu as G
    batch = G.Batch([_spec("sq64_mg3", "fp64"), _spec("sq64_mg1_plate", "fp64")], lanes=2)
    st = G.IBState(batch.members[0])
    G.advance(st, batch.members[0], 0.0, nsteps=1)
    with pytest.raises(G.IBPMError):
        batch.advance(1)
    batch.close()


# members of one grid with different Re, dt and bodies: a group of shared
# launches per precision, beside a member of another grid
GROUPED = [("sq64_mg3", "fp64", 40.0, 0.01), ("sq64_mg3", "fp64", 150.0, 0.008), ("sq64_mg3", "fp64", 90.0, 0.01),
           ("sq64_mg3", "fp32_refined", 60.0, 0.01), ("sq64_mg3", "fp32_refined", 200.0, 0.006),
           ("rect64x32_mg2_two", "fp64", 100.0, 0.005)]


@pytest.mark.parametrize("chain,lanes", [(0, 2), (1, 2), (1, 0)])
def test_grouped_members_match_single_runs(chain, lanes):
    """The FP64 and the FP32-refined sq64 members each form a group whose
    transforms and stencils are launches over all its members; every member's
    CD/CL and state are those of its own handle bit for bit, and the same
    batch stepped member by member gives the same bits.  With lanes = 0 the
    tuner may give each group its own transform plan: each member is compared
    with a handle on that member's plan."""
    import ibpm_gpu as G
    specs = []
    for name, prec, re, dt in GROUPED:
        sp = _spec(name, prec)
        sp["Re"], sp["dt"] = re, dt
        specs.append(sp)
    batch = G.Batch(specs, lanes=lanes)
    batch.set_chain(chain)
    runs = {}
    for grouped in (True, False):
        batch.set_grouped(grouped)
        for i, (name, _, _, _) in enumerate(GROUPED):
            _start(batch.members[i], name, seed=60 + i)
        runs[grouped] = (batch.advance(NSTEPS), [G.IBState(m) for m in batch.members])
    forces, states = runs[True]
    for i, (name, prec, re, dt) in enumerate(GROUPED):
        sp = specs[i]
        solo = G.IBProblem(sp["grid"], sp["bodies"], sp["dt"], sp["Re"], freestream=sp["freestream"],
                           precision=prec, sync_fields=False)
        G.set_transform_plan(solo, *G.transform_plan(batch.members[i]))
        G.set_level_chain(solo, chain)
        _start(solo, name, seed=60 + i)
        st = G.IBState(solo)
        cd, cl = G.advance(st, solo, 0.0, nsteps=NSTEPS)
        G.pull_state(st, solo)
        assert np.array_equal(forces[i][0], cd) and np.array_equal(forces[i][1], cl), (name, prec, re)
        assert np.array_equal(states[i].Gamma, st.Gamma) and np.array_equal(states[i].q, st.q), (name, prec, re)
        f1, s1 = runs[False][0][i], runs[False][1][i]
        assert np.array_equal(f1[0], cd) and np.array_equal(s1.Gamma, st.Gamma), (name, prec, re)
        solo.close()
    batch.close()


def test_batch_member_is_released_with_its_batch():
    import ibpm_gpu as G
    batch = G.Batch([_spec("sq64_mg3", "fp64"), _spec("sq64_mg3", "fp64")], lanes=1)
    m = batch.members[0]
    assert m.lib.ibpm_destroy(m.handle) == G.IBPM_ERR_INVALID
    batch.advance(2)
    batch.close()
