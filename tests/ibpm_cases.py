"""Problem definitions shared by the parity tests and the golden-fixture
generator.  Each case is built identically for the oracle and for the GPU."""
import numpy as np

CASES = {
    # square grid, three nested levels, one cylinder
    "sq64_mg3": dict(h=0.0625, bnd=(-2.0, 2.0, -2.0, 2.0), mg=3, Re=40.0, dt=0.01,
                     bodies=[("cyl", 0.5, 0.0, 0.0, 40)], fs=(1.0, 0.0, 0.0)),
    # rectangular grid (nx != ny), two bodies, inclined freestream
    "rect64x32_mg2_two": dict(h=0.0625, bnd=(-2.0, 2.0, -1.0, 1.0), mg=2, Re=100.0, dt=0.005,
                              bodies=[("cyl", 0.25, -0.5, 0.0, 20), ("cyl", 0.25, 0.5, 0.1, 20)],
                              fs=(1.0, 0.2, 0.1)),
    # single grid, a flat plate
    "sq64_mg1_plate": dict(h=0.0625, bnd=(-2.0, 2.0, -2.0, 2.0), mg=1, Re=200.0, dt=0.01,
                           bodies=[("plate", 1.0, 0.2, -0.5, 0.1, 17)], fs=(1.0, 0.0, 0.0)),
    # 200x200, h=0.02, 3 levels, 157-point cylinder, Re=40, dt=0.004
    "cyl200_mg3": dict(h=0.02, bnd=(-1.0, 3.0, -2.0, 2.0), mg=3, Re=40.0, dt=0.004,
               bodies=[("cyl", 0.5, 0.0, 0.0, 157)], fs=(1.0, 0.0, 0.0)),
}


def build_bodies(mod, spec, h):
    out = []
    for b in spec:
        if b[0] == "cyl":
            _, r, x0, y0, n = b
            out.append(mod.make_cylinder(r, h, x0, y0, n=n))
        else:
            _, L, a, x0, y0, n = b
            out.append(mod.make_plate(L, a, h, x0, y0, n=n))
    return out


def oracle_problem(name):
    from oracle import ibpm_ref as R
    c = CASES[name]
    g = R.make_grid(c["h"], c["bnd"], c["mg"])
    Ux, Uy, a = c["fs"]
    return R.IBProblem(grid=g, bodies=build_bodies(R, c["bodies"], g.h), dt=c["dt"], Re=c["Re"],
                       Ux=Ux, Uy=Uy, inclination=a)


def gpu_problem(name, **kw):
    import ibpm_gpu as G
    c = CASES[name]
    g = G.make_grid(c["h"], c["bnd"], c["mg"])
    return G.IBProblem(g, build_bodies(G, c["bodies"], g.h), c["dt"], c["Re"], freestream=c["fs"], **kw)


def random_state(prob, seed, amp=1e-3):
    """A seeded oracle state: random Γ on every level, ψ and q from vort2flux
    (so Γ is coarsified), random previous nonlinear term."""
    from oracle import ibpm_ref as R
    rng = np.random.default_rng(seed)
    st = R.make_state(prob)
    st.Gamma = amp * rng.standard_normal(st.Gamma.shape)
    R.refresh_flux(st, prob)
    st.nonlin[1] = amp * rng.standard_normal(st.Gamma.shape)
    st.nonlin[0] = st.nonlin[1].copy()
    return st


def to_gpu_state(ost, gst):
    """Copy an oracle state into a GPU host mirror (reference layouts)."""
    from oracle import ibpm_ref as R
    gst.Gamma[:] = R.gamma_to_ref(ost.Gamma)
    gst.psi[:] = R.gamma_to_ref(ost.psi)
    gst.q[:] = R.flux_to_ref(ost.qx, ost.qy)
    gst.q0[:] = R.flux_to_ref(ost.q0x, ost.q0y)
    gst.nonlin[0][:] = R.gamma_to_ref(ost.nonlin[0])
    gst.nonlin[1][:] = R.gamma_to_ref(ost.nonlin[1])
    gst.Fb[:, 0] = ost.Fb


def rel(a, b):
    b = np.asarray(b)
    d = np.max(np.abs(np.asarray(a) - b))
    s = np.max(np.abs(b))
    return d / s if s > 0 else d


# A body point exactly on a grid line puts δh samples exactly at |r| = h, 2h,
# 3h, where the reference's smoothed delta (rounded 10-digit coefficients,
# interface-coupling.jl:32-56) jumps by up to 3e-9: which side a sample takes
# depends on the last bit of r.  Cylinders centred on grid nodes have such
# points; shifting a body by OFF_GRID (a few 1e-7, not a multiple of h) moves
# every point off the grid lines.
OFF_GRID = (1.234e-7, -0.711e-7)


def ulp_moved_body(mod, body):
    """The same body with every point moved by one ulp (towards +inf)."""
    return mod.Body(xb=np.nextafter(body.xb, np.inf), ds=body.ds.copy()) if hasattr(mod, "Body") else \
        mod.RigidBody(xb=np.nextafter(body.xb, np.inf), ds=body.ds.copy())


def force_scale_err(cl, ocl, ocd):
    """max |CL − CL_oracle| over max |CD_oracle|: the lift error on the force
    scale (the lift of a symmetric start is many orders below the drag)."""
    return float(np.max(np.abs(np.asarray(cl) - np.asarray(ocl))) / np.max(np.abs(np.asarray(ocd))))
