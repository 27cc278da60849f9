"""The oracle's moving-grid base flux (base_flux! for a MovingGrid,
timestepping.jl:273-318, with the face coordinates of models.jl:135-153) and
the committed golden force history of the reference's pitch manoeuvre."""
import json
import math
import os

import numpy as np

from ibpm_cases import CASES, build_bodies

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "eldredge_pitch.json")


def _plate_problem(motion=None, fs=(0.0, 0.0, 0.0), name="sq64_mg1_plate", mg=None):
    from oracle import ibpm_ref as R
    c = CASES[name]
    g = R.make_grid(c["h"], c["bnd"], mg or c["mg"])
    return R.IBProblem(grid=g, bodies=build_bodies(R, c["bodies"], g.h), dt=c["dt"], Re=c["Re"],
                       Ux=fs[0], Uy=fs[1], inclination=fs[2], motion=motion)


def test_face_coordinates_are_the_level_centres():
    """Level 1 faces sit at (j − ½) h − offy; every coarser level keeps the
    domain centre and doubles the spacing."""
    from oracle import ibpm_ref as R
    g = R.make_grid(0.0625, (-1.0, 3.0, -2.0, 2.0), 3)
    XX, YY = R.moving_grid_coords(g, 0.0, 0.0)
    assert np.allclose(YY[0], (np.arange(1, g.ny + 1) - 0.5) * g.h - g.offy, rtol=0, atol=1e-14)
    assert np.allclose(XX[0], (np.arange(1, g.nx + 1) - 0.5) * g.h - g.offx, rtol=0, atol=1e-14)
    cx, cy = g.nx / 2 * g.h - g.offx, g.ny / 2 * g.h - g.offy
    for lev in range(g.mg):
        assert abs(XX[lev].mean() - cx) < 1e-13 and abs(YY[lev].mean() - cy) < 1e-13
        assert np.allclose(np.diff(XX[lev]), g.hc(lev)) and np.allclose(np.diff(YY[lev]), g.hc(lev))
    X2, Y2 = R.moving_grid_coords(g, 0.25, -0.5)
    assert np.allclose(X2, XX - 0.25) and np.allclose(Y2, YY + 0.5)


def test_base_flux_is_rotation_plus_translation():
    """The circulation C'q0 of the base flux is the solid-body rotation's,
    2Ω hc² in every cell of every level, and q0 averages to hc (Ux0, Uy0) about
    the grid centre."""
    from oracle import ibpm_ref as R
    mot = R.MovingGrid(U=lambda t: 1.0, V=lambda t: 0.3, theta=lambda t: 0.2 * t, theta_dot=lambda t: 0.2)
    p = _plate_problem(mot, mg=3, fs=(0.5, 0.0, 0.1))
    t = 0.7
    Om, Ux0, Uy0 = R.moving_grid_rates(p, t)
    assert Om == -0.2
    a = -0.2 * t
    assert abs(Ux0 - (math.cos(a) - 0.3 * math.sin(a) + 0.5 * math.cos(0.1))) < 1e-15
    assert abs(Uy0 - (math.sin(a) + 0.3 * math.cos(a) + 0.5 * math.sin(0.1))) < 1e-15
    q0x, q0y = R.base_flux(p, t)
    g = p.grid
    for lev in range(g.mg):
        hc = g.hc(lev)
        G = R.rot(q0x[lev], q0y[lev], g)
        assert np.allclose(G, 2 * Om * hc * hc, rtol=1e-12, atol=0)
        # the grid centre is (0, 0) here, so the face averages are the translation
        assert abs(q0x[lev].mean() - hc * Ux0) < 1e-13 and abs(q0y[lev].mean() - hc * Uy0) < 1e-13


def test_non_rotating_moving_grid_is_the_static_problem():
    """MovingGrid(U, V, θ ≡ −i, θ̇ ≡ 0) with no free stream of its own is the
    static problem in the free stream (U, V, inclination i), to the bit."""
    from oracle import ibpm_ref as R
    U, V, inc = 1.0, 0.2, 0.15
    mot = R.MovingGrid(U=lambda t: U, V=lambda t: V, theta=lambda t: -inc, theta_dot=lambda t: 0.0)
    pm = _plate_problem(mot)
    ps = _plate_problem(None, fs=(U, V, inc))
    sm, ss = R.make_state(pm), R.make_state(ps)
    assert np.array_equal(sm.q0x, ss.q0x) and np.array_equal(sm.q0y, ss.q0y)
    cdm, clm = R.run(pm, sm, 5)
    cds, cls = R.run(ps, ss, 5)
    assert np.array_equal(cdm, cds) and np.array_equal(clm, cls)
    assert np.array_equal(sm.Gamma, ss.Gamma)


def test_moving_grid_step_uses_the_motion_at_t():
    """advance(state, prob, t) recomputes q0 from the motion at t before the
    trial step (timestepping.jl:41-43): two runs started at different t differ
    exactly by the motion's time shift."""
    from oracle import ibpm_ref as R
    mot = R.MovingGrid(U=lambda t: 1.0, V=lambda t: 0.0, theta=lambda t: 0.3 * math.sin(2 * t),
                       theta_dot=lambda t: 0.6 * math.cos(2 * t))
    shifted = R.MovingGrid(U=lambda t: 1.0, V=lambda t: 0.0, theta=lambda t: 0.3 * math.sin(2 * (t + 0.4)),
                           theta_dot=lambda t: 0.6 * math.cos(2 * (t + 0.4)))
    p1, p2 = _plate_problem(mot), _plate_problem(shifted)
    s1, s2 = R.make_state(p1), R.make_state(p2)
    c1 = R.run(p1, s1, 4, t0=0.4)
    c2 = R.run(p2, s2, 4, t0=0.0)
    assert np.allclose(c1[0], c2[0], rtol=1e-12, atol=1e-15)
    q0x, _ = R.base_flux(p1, 0.4 + 3 * p1.dt)
    assert np.array_equal(s1.q0x, q0x)


def eldredge_motion():
    """θ(t), θ̇(t) of the reference's pitch manoeuvre
    (benchmarks/eldredge/pitch_maneuver.jl:11-20): a = 11, t1..t4 = 1, 3, 4, 6,
    α_max = 45°, G normalised by its maximum over t = 0:1e-3:10."""
    a = 11.0
    t1, t2, t3, t4 = 1.0, 3.0, 4.0, 6.0
    amax = 45 * math.pi / 180

    def G(t):
        return np.log(np.cosh(a * (t - t1)) * np.cosh(a * (t - t4)) / (np.cosh(a * (t - t2)) * np.cosh(a * (t - t3))))

    def Gd(t):
        return a * (np.tanh(a * (t - t1)) - np.tanh(a * (t - t2)) - np.tanh(a * (t - t3)) + np.tanh(a * (t - t4)))

    gmax = float(np.max(G(np.arange(10001) * 1e-3)))
    return (lambda t: float(-amax * G(t) / gmax)), (lambda t: float(-amax * Gd(t) / gmax))


def test_eldredge_golden_fixture():
    """The committed force history: t = 0:0.01:10, the first sample is the
    steady plate's drag (the published 0.39415052 to the fixture's digits) at
    zero lift, and the lift peaks during the pitch-up, where θ is near −45°."""
    with open(GOLDEN) as f:
        d = json.load(f)
    t = np.array(d["t"])
    cl, cd = np.array(d["CL_lab"]), np.array(d["CD_lab"])
    assert t.size == 1001 and np.allclose(t, np.arange(1001) * 0.01, rtol=0, atol=1e-12)
    assert abs(cd[0] - d["steady_cd_published"]["julia"]) < 2e-8 and abs(cl[0]) < 1e-6
    theta, _ = eldredge_motion()
    tpk = t[np.argmax(cl)]
    assert 1.0 < tpk < 4.0 and theta(tpk) < -0.5
    assert abs(theta(3.5) + math.pi / 4) < 1e-6
