"""Moving grid (MovingGrid, base_flux! of timestepping.jl:273-318) on the GPU
through the C ABI: against the oracle on small pitching problems, and against
the reference's own force history of the pitch manoeuvre of
benchmarks/eldredge (golden/eldredge_pitch.json)."""
import json
import math
import os

import numpy as np
import pytest

from ibpm_cases import CASES, build_bodies, random_state, rel, to_gpu_state
from test_moving_grid_oracle import GOLDEN, eldredge_motion

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _motions(mod):
    return mod.MovingGrid(U=lambda t: 1.0, V=lambda t: 0.1, theta=lambda t: 0.3 * math.sin(2 * t),
                          theta_dot=lambda t: 0.6 * math.cos(2 * t))


def _pair(name, mg=None, precision="fp64", refine_sweeps=1, fs=(0.2, 0.0, 0.05)):
    import ibpm_gpu as G
    from oracle import ibpm_ref as R
    c = CASES[name]
    og = R.make_grid(c["h"], c["bnd"], mg or c["mg"])
    ob = build_bodies(R, c["bodies"][:1], og.h)
    op = R.IBProblem(grid=og, bodies=ob, dt=c["dt"], Re=c["Re"], Ux=fs[0], Uy=fs[1], inclination=fs[2],
                     motion=_motions(R))
    gg = G.make_grid(c["h"], c["bnd"], mg or c["mg"])
    gb = build_bodies(G, c["bodies"][:1], gg.h)
    gb[0].motion = _motions(G)
    gp = G.IBProblem(gg, gb, c["dt"], c["Re"], freestream=fs, precision=precision, refine_sweeps=refine_sweeps)
    return op, gp


@pytest.mark.parametrize("name,mg", [("sq64_mg1_plate", 1), ("sq64_mg1_plate", 3), ("rect64x32_mg2_two", 2)])
@pytest.mark.parametrize("nsteps", [1, 15])
def test_moving_grid_matches_oracle(name, mg, nsteps):
    import ibpm_gpu as G
    from oracle import ibpm_ref as R
    op, gp = _pair(name, mg)
    ost = random_state(op, seed=40 + nsteps)
    gst = G.IBState(gp)
    # before any step q0 is the base flux at t = 0 (IBState calls base_flux!)
    q0x, q0y = R.base_flux(op, 0.0)
    assert rel(gst.q0, R.flux_to_ref(q0x, q0y)) < 1e-15
    to_gpu_state(ost, gst)
    G.push_state(gst, gp)
    t0 = 0.35
    cd, cl = G.advance(gst, gp, t0, nsteps=nsteps)
    ocd, ocl = R.run(op, ost, nsteps, t0=t0)
    assert rel(gst.Gamma, R.gamma_to_ref(ost.Gamma)) < TOL
    assert rel(gst.psi, R.gamma_to_ref(ost.psi)) < TOL
    assert rel(gst.q, R.flux_to_ref(ost.qx, ost.qy)) < TOL
    assert rel(gst.nonlin[0], R.gamma_to_ref(ost.nonlin[0])) < TOL
    assert rel(gst.Fb[:, 0], ost.Fb) < TOL
    assert rel(cd, ocd) < TOL and rel(cl, ocl) < TOL
    # q0 reported is the last step's base flux
    assert rel(gst.q0, R.flux_to_ref(ost.q0x, ost.q0y)) < 1e-15
    gp.close()


def test_moving_grid_refined_matches_oracle():
    import ibpm_gpu as G
    from oracle import ibpm_ref as R
    op, gp = _pair("sq64_mg1_plate", 3, precision="fp32_refined", refine_sweeps=2)
    ost = random_state(op, seed=5)
    gst = G.IBState(gp)
    to_gpu_state(ost, gst)
    G.push_state(gst, gp)
    cd, cl = G.advance(gst, gp, 0.1, nsteps=15)
    ocd, ocl = R.run(op, ost, 15, t0=0.1)
    assert rel(gst.Gamma, R.gamma_to_ref(ost.Gamma)) < 1e-9
    assert rel(cd, ocd) < 1e-9 and rel(cl, ocl) < 1e-9
    gp.close()


def test_non_rotating_moving_grid_is_the_static_problem():
    """MovingGrid(U, V, θ ≡ −i, θ̇ ≡ 0) without a free stream of its own steps
    as the static problem in the free stream (U, V, i): the same base flux to
    the bit, the same step to rounding (the moving form is its own kernel
    instantiation, whose multiply-adds the compiler may fuse differently)."""
    import ibpm_gpu as G
    c = CASES["sq64_mg3"]
    U, V, inc = 1.0, 0.2, 0.15
    g = G.make_grid(c["h"], c["bnd"], c["mg"])
    bm = build_bodies(G, c["bodies"], g.h)
    bm[0].motion = G.MovingGrid(U=lambda t: U, V=lambda t: V, theta=lambda t: -inc, theta_dot=lambda t: 0.0)
    pm = G.IBProblem(g, bm, c["dt"], c["Re"], freestream=(0.0, 0.0, 0.0))
    ps = G.IBProblem(g, build_bodies(G, c["bodies"], g.h), c["dt"], c["Re"], freestream=(U, V, inc))
    sm, ss = G.IBState(pm), G.IBState(ps)
    assert np.array_equal(sm.q0, ss.q0)
    cdm, clm = G.advance(sm, pm, 0.0, nsteps=20)
    cds, cls = G.advance(ss, ps, 0.0, nsteps=20)
    assert rel(cdm, cds) < 1e-13 and rel(clm, cls) < 1e-13
    assert rel(sm.Gamma, ss.Gamma) < 1e-13 and rel(sm.q, ss.q) < 1e-13
    pm.close()
    ps.close()


def test_moving_grid_refusals():
    import ibpm_gpu as G
    op, gp = _pair("sq64_mg1_plate", 2)
    # stepping without the motion, the adjoint and batches refuse a moving grid
    with pytest.raises(G.IBPMError):
        gp._check(gp.lib.ibpm_advance(gp.handle, 0.0, 1, None, None))
    with pytest.raises(G.IBPMError):
        G.adjoint_run(gp, 4, k_checkpoint=2)
    gp.close()
    c = CASES["rect64x32_mg2_two"]
    g = G.make_grid(c["h"], c["bnd"], c["mg"])
    bodies = build_bodies(G, c["bodies"], g.h)
    bodies[0].motion = _motions(G)
    with pytest.raises(G.IBPMError):                # one body only (models.jl:137)
        G.IBProblem(g, bodies, c["dt"], c["Re"], freestream=(0.0, 0.0, 0.0))


def _eldredge_grid(G):
    return G.make_grid(0.02, (-1.5, 6.5, -2.0, 2.0), 5)


def test_eldredge_pitch_manoeuvre_against_reference_history():
    """benchmarks/eldredge: the steady flat-plate boundary layer
    (steady_bl.jl: 400×200 × 5 levels, Re = 100, 51 points, dt = 0.01,
    t = 0:0.01:100) and from it the moving-grid pitch-up-hold-down
    (pitch_maneuver.jl: dt = 1e-3, t = 0:1e-3:10, α_max = 45°), lab-frame
    CL, CD against the reference's force_jl2.mat history."""
    import ibpm_gpu as G
    with open(GOLDEN) as f:
        gold = json.load(f)
    g = _eldredge_grid(G)
    plate = G.make_plate(1.0, 0.0, g.h, 0.0, 0.0, n=51)
    steady = G.IBProblem(g, [plate], 1e-2, 100.0, freestream=(1.0, 0.0, 0.0), sync_fields=False)
    st = G.IBState(steady)
    cd, cl = G.advance(st, steady, np.arange(10001) * 1e-2)
    # published: Julia 0.39415052, Fortran 0.39415060 (benchmarks/eldredge/README.md:25-26)
    assert abs(cd[-1, 0] - gold["steady_cd_published"]["julia"]) < 2e-8, cd[-1, 0]
    G.pull_state(st, steady)
    steady.close()

    theta, theta_dot = eldredge_motion()
    plate_m = G.make_plate(1.0, 0.0, g.h, 0.0, 0.0, n=51,
                           motion=G.MovingGrid(U=lambda t: 1.0, V=lambda t: 0.0, theta=theta, theta_dot=theta_dot))
    pitch = G.IBProblem(g, [plate_m], 1e-3, 100.0, freestream=(0.0, 0.0, 0.0), sync_fields=False)
    G.push_state(st, pitch)
    t = np.arange(10001) * 1e-3
    F1, F2 = G.advance(st, pitch, t)
    th = np.array([theta(tk) for tk in t])
    CD = F1[:, 0] * np.cos(th) - F2[:, 0] * np.sin(th)
    CL = F1[:, 0] * np.sin(th) + F2[:, 0] * np.cos(th)
    k = gold["step_stride"]
    gcl, gcd = np.array(gold["CL_lab"]), np.array(gold["CD_lab"])
    ecl = np.max(np.abs(CL[::k] - gcl)) / np.max(np.abs(gcl))
    ecd = np.max(np.abs(CD[::k] - gcd)) / np.max(np.abs(gcd))
    out = os.environ.get("IBPM_ELDREDGE_OUT")
    if out:
        np.savez(out, t=t, CL=CL, CD=CD, F1=F1[:, 0], F2=F2[:, 0])
    print("eldredge: max |CL - ref| / max|CL_ref| = %.3e, CD: %.3e" % (ecl, ecd))
    # observed: 1.2e-9 (CL) and 1.3e-9 (CD) of the peak over the whole history
    assert ecl < 1e-8 and ecd < 1e-8, (ecl, ecd)
    pitch.close()
