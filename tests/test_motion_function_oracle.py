"""The oracle's MotionFunction bodies (move_body!, move-body-utils.jl:86-133;
update_bodies!, timestepping.jl:386-398; boundary_forces!, :174-186) and the
committed force history of the reference's moving-body pitch manoeuvre."""
import json
import math
import os

import numpy as np

from ibpm_cases import CASES, build_bodies

GOLDEN_MOTION = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "eldredge_pitch_motion.json")


def _plate(motion=None, mg=2):
    from oracle import ibpm_ref as R
    c = CASES["sq64_mg1_plate"]
    g = R.make_grid(c["h"], c["bnd"], mg)
    bodies = build_bodies(R, c["bodies"], g.h)
    return R.IBProblem(grid=g, bodies=bodies, dt=c["dt"], Re=c["Re"], motion=motion)


def test_still_motion_function_is_the_static_problem():
    """A MotionFunction that stays at the reference configuration steps as the
    static body, to the bit (E and B⁻¹ rebuilt from the same points)."""
    from oracle import ibpm_ref as R
    zero = (lambda t: 0.0,) * 3
    ps, pm = _plate(), _plate([R.MotionFunction(xc=zero, uc=zero)])
    ss, sm = R.make_state(ps), R.make_state(pm)
    a = R.run(ps, ss, 4)
    b = R.run(pm, sm, 4)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    assert np.array_equal(ss.Gamma, sm.Gamma)


def test_rigid_motion_velocity_is_the_time_derivative():
    """ub = vel + Ru x0 is d/dt of xb = pos + Rx x0 when uc = d(xc)/dt."""
    from oracle import ibpm_ref as R
    m = R.MotionFunction(xc=(lambda t: 0.1 * math.sin(t), lambda t: -0.2 * t, lambda t: 0.4 * math.cos(3 * t)),
                         uc=(lambda t: 0.1 * math.cos(t), lambda t: -0.2, lambda t: -1.2 * math.sin(3 * t)))
    x0 = np.random.default_rng(1).standard_normal((9, 2))
    t, eps = 0.37, 1e-6
    _, ub = R.rigid_motion(m, x0, t)
    xp, _ = R.rigid_motion(m, x0, t + eps)
    xm, _ = R.rigid_motion(m, x0, t - eps)
    assert np.allclose(ub, (xp - xm) / (2 * eps), rtol=0, atol=1e-8)
    xb, _ = R.rigid_motion(m, x0, 0.0)
    th = 0.4
    rot = np.array([[math.cos(th), -math.sin(th)], [math.sin(th), math.cos(th)]])
    assert np.allclose(xb, x0 @ rot.T, rtol=0, atol=1e-15)


def test_moving_body_enforces_the_body_velocity():
    """After a step the regularised flux at the points is the body velocity:
    E(q + q0) = ub·h (the constraint boundary_forces! solves for)."""
    from oracle import ibpm_ref as R
    m = R.MotionFunction(xc=(lambda t: 0.0, lambda t: 0.05 * math.sin(4 * t), lambda t: 0.0),
                         uc=(lambda t: 0.0, lambda t: 0.2 * math.cos(4 * t), lambda t: 0.0))
    p = _plate([m], mg=1)
    st = R.make_state(p)
    R.run(p, st, 3, t0=0.2)
    F = R.E_apply(st.qx[0] + st.q0x[0], st.qy[0] + st.q0y[0], p)
    ub = np.concatenate([p.ub[:, 0], p.ub[:, 1]]) * p.grid.h
    assert np.max(np.abs(F - ub)) <= 1e-10 * max(1.0, np.max(np.abs(F)))


def test_moving_body_golden_fixture():
    """force_jl1.mat: t = 0:0.01:9.99, the first sample is the steady plate's
    drag at zero lift; it differs from the moving-grid history (force_jl2.mat)
    by about 1% at the lift peak (the two formulations)."""
    with open(GOLDEN_MOTION) as f:
        d = json.load(f)
    t = np.array(d["t"])
    assert t.size == 1000 and np.allclose(t, np.arange(1000) * 0.01, rtol=0, atol=1e-12)
    assert abs(d["CD_lab"][0] - 0.39415052) < 2e-8 and abs(d["CL_lab"][0]) < 1e-6
    with open(GOLDEN_MOTION.replace("_motion", "")) as f:
        g = json.load(f)
    dcl = np.max(np.abs(np.array(d["CL_lab"]) - np.array(g["CL_lab"][:1000]))) / np.max(np.abs(g["CL_lab"]))
    assert 1e-3 < dcl < 5e-2
