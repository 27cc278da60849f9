"""The Python usage example that the integration guide quotes: the calls a user of
the ctypes mirror makes for each feature.  tests/test_gpu_integration_doc.py
runs it and checks what it leaves behind; run from the repository root as
`python tests/integration_example.py` it needs a B200 and the built library."""
import os
import sys

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "ibpm.jl_b200", "python"))
import math
import numpy as np
import ibpm_gpu as G

g = G.make_grid(0.01, (-1.0, 4.12, -2.56, 2.56), 5)              # 512 x 512 cells, 5 levels
cyl = lambda: G.make_cylinder(0.5, g.h, 0.0, 0.0, n=314)
prob = G.IBProblem(g, [cyl()], 0.002, 100.0)                      # free stream (1, 0, 0)
state = G.IBState(prob)
cd, cl = G.advance(state, prob, 0.0, nsteps=1000)                 # advance!, 1000 times

# FP32-refined form and the discrete adjoint
prob32 = G.IBProblem(g, [cyl()], 0.002, 100.0, precision="fp32_refined")
res = G.adjoint_run(prob32, 1000, k_checkpoint=50, window=200)    # res.J, res.grad_omega0, res.grad_alpha
res = G.adjoint_run(prob, 200, 100, 100, w_cd=0.0, w_cl=1.0, want_xb=True)   # res.grad_xb: (nb, 2)

# a moving grid: one body, base flux from the motion at each step's t
theta = lambda t: -0.5 * math.sin(t)
theta_dot = lambda t: -0.5 * math.cos(t)
mot = G.MovingGrid(U=lambda t: 1.0, V=lambda t: 0.0, theta=theta, theta_dot=theta_dot)
pp = G.IBProblem(g, [G.make_plate(1.0, 0.0, g.h, 0.0, 0.0, n=51, motion=mot)], 1e-3, 100.0,
                 freestream=(0.0, 0.0, 0.0))
F1, F2 = G.advance(G.IBState(pp), pp, np.arange(1000) * 1e-3)     # body-frame CD, CL per step

# a moving body: the plate itself pitches (E and B⁻¹ rebuilt every step)
mf = G.MotionFunction(xc=(lambda t: 0.0, lambda t: 0.0, theta), uc=(lambda t: 0.0, lambda t: 0.0, theta_dot))
pb = G.IBProblem(g, [G.make_plate(1.0, 0.0, g.h, 0.0, 0.0, n=51, motion=mf)], 1e-3, 100.0)
CD, CL = G.advance(G.IBState(pb), pb, np.arange(100) * 1e-3)      # lab-frame CD, CL per step
xb, ub = G.body_points(pb)                                        # state.xb and the points' velocities

# many independent simulations, one graph launch per step (one grid here:
# every transform and stencil of a step is one launch over all three)
batch = G.Batch([dict(grid=g, bodies=[cyl()], dt=0.002, Re=Re) for Re in (40.0, 100.0, 200.0)])
histories = batch.advance(1000)                                   # [(CD, CL)] per member
