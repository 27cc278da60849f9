"""Python host mirror of IBPM.jl's interface over libibpm_gpu.so (ctypes).

The reference's user-facing pieces for the static-body time step are kept,
with the same names and argument meanings:

* ``make_grid(h, boundary, mg)``       src/fluid-domain/fluid-domain.jl:44-73
* ``make_cylinder``, ``make_plate``, ``make_naca``
                                       src/structure-domain/sample-bodies.jl:17-134
* ``IBProblem(grid, bodies, dt, Re, freestream=...)``
                                       src/pre-processing/problem-types.jl:23-41
* ``MovingGrid(U, V, theta, theta_dot)`` src/structure-domain/motion-types.jl:40-48
* ``MotionFunction(xc, uc)``            src/structure-domain/motion-types.jl:13-17
* ``IBState(prob)``                    src/pre-processing/state-types.jl:25-47
* ``advance(state, prob, t)``          advance!(state, prob, t), src/timestepping/timestepping.jl:35-67
* ``vort2flux(state, prob)``           vort2flux!(ψ, q, Γ, model, mg), src/fluid-operators/curl.jl:133-165

All arrays use the reference's shapes and column-major layouts (``order='F'``
views are not needed: ``state.Gamma`` is the (nΓ, mg) matrix flattened by
column, exactly ``vec`` of the Julia matrix).  Every compute call runs in the
CUDA library; there is no CPU fallback: if the library or a GPU is missing,
the calls raise ``IBPMError``.
"""
from __future__ import annotations

import ctypes as C
import math
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.normpath(os.path.join(_HERE, "..", "..", "lib", "libibpm_gpu.so"))
HEADER_PATH = os.path.normpath(os.path.join(_HERE, "..", "..", "..", "include", "ibpm_gpu.h"))

IBPM_OK = 0
IBPM_ERR_INVALID = -1
IBPM_ERR_CUDA = -2
IBPM_ERR_NONFINITE = -3
IBPM_ERR_UNSUPPORTED = -4
IBPM_ERR_NOMEM = -5
IBPM_PREC_FP64 = 0
IBPM_PREC_FP32_REFINED = 1
# transform plans (ibpm_set_transform_plan): radix 4 / N/4 threads per line
# pair (shortest chain per launch), radix 8 / N/8 threads (fewer instructions)
IBPM_PLAN_LATENCY = 0
IBPM_PLAN_THROUGHPUT = 1
IBPM_PLAN_AUTO = 2      # multi-slab launches: throughput plan from 4 slabs on
# level chains of vort2flux! (ibpm_set_level_chain): the reference's order, one
# level after another, or the boundary transfer (all levels per launch)
IBPM_CHAIN_SEQUENTIAL = 0
IBPM_CHAIN_BOUNDARY_TRANSFER = 1
PRECISIONS = {"fp64": IBPM_PREC_FP64, "fp32_refined": IBPM_PREC_FP32_REFINED}
KERNEL_COUNT = 12

_ERRNAMES = {IBPM_ERR_INVALID: "INVALID", IBPM_ERR_CUDA: "CUDA", IBPM_ERR_NONFINITE: "NONFINITE",
             IBPM_ERR_UNSUPPORTED: "UNSUPPORTED", IBPM_ERR_NOMEM: "NOMEM"}


class IBPMError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("ibpm error %d (%s): %s" % (code, _ERRNAMES.get(code, "?"), msg))
        self.code = code


class ProblemDesc(C.Structure):
    """Mirror of ``ibpm_problem_desc`` in include/ibpm_gpu.h."""
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("mg", C.c_int32),
                ("h", C.c_double), ("offx", C.c_double), ("offy", C.c_double),
                ("Re", C.c_double), ("dt", C.c_double),
                ("Ux", C.c_double), ("Uy", C.c_double), ("inclination", C.c_double),
                ("beta", C.c_double * 2),
                ("nbodies", C.c_int32), ("nb", C.c_int32),
                ("body_npts", C.POINTER(C.c_int32)), ("xb", C.POINTER(C.c_double)),
                ("ds", C.POINTER(C.c_double)),
                ("precision", C.c_int32), ("device", C.c_int32), ("refine_sweeps", C.c_int32)]


class Objective(C.Structure):
    """Mirror of ``ibpm_objective``: J = (1/window) Σ over the last ``window``
    steps of Σ_bodies (w_cd CD + w_cl CL)."""
    _fields_ = [("window", C.c_int32), ("w_cd", C.c_double), ("w_cl", C.c_double)]


_DP = C.POINTER(C.c_double)
_lib = None


def load_library(path=None):
    """Load libibpm_gpu.so (built in-tree by ``make -C ibpm.jl_b200/csrc``)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise IBPMError(IBPM_ERR_INVALID, "CUDA library not built: %s (run make -C ibpm.jl_b200/csrc)" % p)
    lib = C.CDLL(p)
    H = C.c_void_p
    lib.ibpm_version.restype = C.c_char_p
    lib.ibpm_version.argtypes = []
    lib.ibpm_create.restype = C.c_int
    lib.ibpm_create.argtypes = [C.POINTER(ProblemDesc), C.POINTER(H)]
    lib.ibpm_destroy.restype = C.c_int
    lib.ibpm_destroy.argtypes = [H]
    lib.ibpm_last_error.restype = C.c_char_p
    lib.ibpm_last_error.argtypes = [H]
    lib.ibpm_sizes.restype = C.c_int
    lib.ibpm_sizes.argtypes = [H, C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.POINTER(C.c_int32),
                               C.POINTER(C.c_int32), C.POINTER(C.c_int32)]
    lib.ibpm_set_state.restype = C.c_int
    lib.ibpm_set_state.argtypes = [H] + [_DP] * 7
    lib.ibpm_set_base_state.restype = C.c_int
    lib.ibpm_set_base_state.argtypes = [H, _DP, _DP]
    lib.ibpm_get_state.restype = C.c_int
    lib.ibpm_get_state.argtypes = [H] + [_DP] * 7
    lib.ibpm_advance.restype = C.c_int
    lib.ibpm_advance.argtypes = [H, C.c_double, C.c_int32, _DP, _DP]
    lib.ibpm_set_moving_grid.restype = C.c_int
    lib.ibpm_set_moving_grid.argtypes = [H, C.c_double, C.c_double, _DP]
    lib.ibpm_advance_moving.restype = C.c_int
    lib.ibpm_advance_moving.argtypes = [H, C.c_int32, _DP, _DP, _DP]
    lib.ibpm_set_motion_function.restype = C.c_int
    lib.ibpm_set_motion_function.argtypes = [H]
    lib.ibpm_advance_bodies.restype = C.c_int
    lib.ibpm_advance_bodies.argtypes = [H, C.c_int32, _DP, _DP, _DP]
    lib.ibpm_get_body_points.restype = C.c_int
    lib.ibpm_get_body_points.argtypes = [H, _DP, _DP]
    lib.ibpm_vort2flux.restype = C.c_int
    lib.ibpm_vort2flux.argtypes = [H]
    lib.ibpm_get_binv.restype = C.c_int
    lib.ibpm_get_binv.argtypes = [H, _DP]
    lib.ibpm_sync.restype = C.c_int
    lib.ibpm_sync.argtypes = [H]
    lib.ibpm_host_alloc.restype = C.c_void_p
    lib.ibpm_host_alloc.argtypes = [C.c_int64]
    lib.ibpm_host_free.restype = C.c_int
    lib.ibpm_host_free.argtypes = [C.c_void_p]
    lib.ibpm_kernel_name.restype = C.c_char_p
    lib.ibpm_kernel_name.argtypes = [C.c_int32]
    lib.ibpm_launches_per_step.restype = C.c_int
    lib.ibpm_launches_per_step.argtypes = [H]
    lib.ibpm_bench.restype = C.c_int
    lib.ibpm_bench.argtypes = [H, C.c_int32, C.c_int32, _DP]
    lib.ibpm_profile.restype = C.c_int
    lib.ibpm_profile.argtypes = [H, C.c_int32, C.c_int32, _DP, _DP, C.POINTER(C.c_int32)]
    lib.ibpm_batch_create.restype = C.c_int
    lib.ibpm_batch_create.argtypes = [C.c_int32, C.POINTER(ProblemDesc), C.c_int32, C.POINTER(H)]
    lib.ibpm_batch_destroy.restype = C.c_int
    lib.ibpm_batch_destroy.argtypes = [H]
    lib.ibpm_batch_member.restype = H
    lib.ibpm_batch_member.argtypes = [H, C.c_int32]
    lib.ibpm_batch_lanes.restype = C.c_int
    lib.ibpm_batch_lanes.argtypes = [H]
    lib.ibpm_batch_plan.restype = C.c_int
    lib.ibpm_batch_plan.argtypes = [H]
    lib.ibpm_batch_set_plan.restype = C.c_int
    lib.ibpm_batch_set_plan.argtypes = [H, C.c_int32]
    lib.ibpm_set_transform_plan.restype = C.c_int
    lib.ibpm_set_transform_plan.argtypes = [H, C.c_int32, C.c_int32]
    lib.ibpm_get_transform_plan.restype = C.c_int
    lib.ibpm_get_transform_plan.argtypes = [H, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]
    lib.ibpm_set_level_chain.restype = C.c_int
    lib.ibpm_set_level_chain.argtypes = [H, C.c_int32]
    lib.ibpm_get_level_chain.restype = C.c_int
    lib.ibpm_get_level_chain.argtypes = [H, C.POINTER(C.c_int32)]
    lib.ibpm_batch_chain.restype = C.c_int
    lib.ibpm_batch_chain.argtypes = [H]
    lib.ibpm_batch_set_chain.restype = C.c_int
    lib.ibpm_batch_set_chain.argtypes = [H, C.c_int32]
    lib.ibpm_batch_grouped.restype = C.c_int
    lib.ibpm_batch_grouped.argtypes = [H]
    lib.ibpm_batch_set_grouped.restype = C.c_int
    lib.ibpm_batch_set_grouped.argtypes = [H, C.c_int32]
    lib.ibpm_batch_set_lanes.restype = C.c_int
    lib.ibpm_batch_set_lanes.argtypes = [H, C.c_int32]
    lib.ibpm_batch_last_error.restype = C.c_char_p
    lib.ibpm_batch_last_error.argtypes = [H]
    lib.ibpm_batch_advance.restype = C.c_int
    lib.ibpm_batch_advance.argtypes = [H, C.c_int32]
    lib.ibpm_batch_get_forces.restype = C.c_int
    lib.ibpm_batch_get_forces.argtypes = [H, C.c_int32, _DP, _DP]
    lib.ibpm_batch_bench.restype = C.c_int
    lib.ibpm_batch_bench.argtypes = [H, C.c_int32, C.c_int32, _DP]
    lib.ibpm_adjoint_run.restype = C.c_int
    lib.ibpm_adjoint_run.argtypes = [H, C.c_int32, C.c_int32, C.POINTER(Objective), _DP, _DP, _DP, _DP, _DP, _DP]
    lib.ibpm_adjoint_bench.restype = C.c_int
    lib.ibpm_adjoint_bench.argtypes = [H, C.c_int32, C.c_int32, _DP]
    if path is None:
        _lib = lib
    return lib


def version():
    return load_library().ibpm_version().decode()


def _ptr(a):
    if a is None:
        return None
    if a.dtype != np.float64 or not (a.flags["C_CONTIGUOUS"] or a.flags["F_CONTIGUOUS"]):
        raise IBPMError(IBPM_ERR_INVALID, "arrays must be contiguous float64")
    return a.ctypes.data_as(_DP)


# --------------------------------------------------------------------------
# Grid and bodies (host-side setup, as in the reference)
# --------------------------------------------------------------------------
@dataclass
class MultiGrid:
    """fluid-domain.jl:10-25."""
    nx: int
    ny: int
    mg: int
    offx: float
    offy: float
    len: float
    h: float

    @property
    def nGamma(self):
        return (self.nx - 1) * (self.ny - 1)

    @property
    def nq(self):
        return self.ny * (self.nx + 1) + self.nx * (self.ny + 1)

    @property
    def nu(self):
        return self.ny * (self.nx + 1)


def make_grid(h, boundary, mg=1):
    """fluid-domain.jl:44-73: nx = round(len/h), ny = round(ylen nx/len), h = len/nx."""
    offx = -boundary[0]
    offy = -boundary[2]
    ln = boundary[1] - boundary[0]
    ylen = boundary[3] - boundary[2]
    nx = int(round(ln / h))
    ny = int(round(ylen * nx / ln))
    return MultiGrid(nx=nx, ny=ny, mg=mg, offx=offx, offy=offy, len=ln, h=ln / nx)


@dataclass
class MovingGrid:
    """MovingGrid (motion-types.jl:40-48): the grid moves with the body.  U, V
    are the lab-frame free stream, theta the body frame's angular position
    (minus the aerodynamic pitch) and theta_dot its rate: callables of t.
    xc, yc are kept for parity; the reference's IBProblem takes the rotational
    flux about the IBModel's (0, 0) (models.jl:127-153), and so does this."""
    U: object
    V: object
    theta: object
    theta_dot: object
    xc: float = 0.0
    yc: float = 0.0

    def row(self, t):
        """(U, V, θ, θ̇) at t."""
        return (float(self.U(t)), float(self.V(t)), float(self.theta(t)), float(self.theta_dot(t)))


@dataclass
class MotionFunction:
    """MotionFunction (motion-types.jl:13-17): the body's points as created are
    its reference configuration, moved rigidly by xc(t) = (x, y, θ) with
    velocity uc(t) = (ẋ, ẏ, θ̇), each a triple of callables
    (move_body!, move-body-utils.jl:86-133)."""
    xc: tuple
    uc: tuple

    def row(self, t):
        """(x, y, θ, ẋ, ẏ, θ̇) at t."""
        return tuple(float(f(t)) for f in self.xc) + tuple(float(f(t)) for f in self.uc)


@dataclass
class RigidBody:
    """RigidBody (body-types.jl:10-16): points xb (nb, 2), ds (nb,) and the
    motion (None: Static; or a MovingGrid)."""
    xb: np.ndarray
    ds: np.ndarray
    motion: object = None


def make_cylinder(r, h, x0, y0, n=0, motion=None):
    """sample-bodies.jl:42-65 (n = 0 chooses ds ≈ 2h)."""
    if n == 0:
        n = int(math.floor(2 * math.pi * r / h / 2))
    spt = np.arange(n) * (2 * math.pi / n)
    xhat = r * np.cos(spt)
    yhat = r * np.sin(spt)
    ds = math.sqrt((xhat[1] - xhat[0]) ** 2 + (yhat[1] - yhat[0]) ** 2)
    return RigidBody(xb=np.stack([xhat + x0, yhat + y0], axis=1), ds=np.full(n, ds), motion=motion)


def make_plate(L, alpha, h, x0, y0, n=0, motion=None):
    """sample-bodies.jl:17-33 (n = 0 chooses ds ≈ 2h)."""
    if n == 0:
        n = int(math.floor(L / h / 2)) + 1
    spt = L * np.arange(n) / (n - 1)
    xhat = spt * math.cos(-alpha)
    yhat = spt * math.sin(-alpha)
    ds = math.sqrt((xhat[1] - xhat[0]) ** 2 + (yhat[1] - yhat[0]) ** 2)
    return RigidBody(xb=np.stack([xhat + x0, yhat + y0], axis=1), ds=np.full(n, ds), motion=motion)


def make_naca(x0, N, t, m=0.0, p=0.0, chord=1.0, aoa=0.0, pivot=(0.0, 0.0), motion=None):
    """sample-bodies.jl:72-134 with a real thickness ``t``, chord scale and a
    rotation by ``aoa`` (rad, nose up) about ``pivot``; panel midpoints and
    lengths as the reference."""
    dth = math.pi / (N - 1)
    x = 0.5 * (1 + np.cos(dth * np.arange(N)))
    yc = np.zeros_like(x)
    th = np.zeros_like(x)
    if m > 0 and p > 0:
        mi = np.nonzero(x < p)[0][-1]
        yc[:mi + 1] = (m / p ** 2) * (2 * p * x[:mi + 1] - x[:mi + 1] ** 2)
        yc[mi + 1:] = (m / (1 - p) ** 2) * (1 - 2 * p + 2 * p * x[mi + 1:] - x[mi + 1:] ** 2)
        dyc = np.zeros_like(x)
        dyc[:mi + 1] = (2 * m / p ** 2) * (p - x[:mi + 1])
        dyc[mi + 1:] = (2 * m / (1 - p ** 2)) * (p - x[mi + 1:])
        th = np.arctan(dyc)
    yt = 5 * t * (0.2969 * np.sqrt(x) - 0.1260 * x - 0.3516 * x ** 2 + 0.2843 * x ** 3 - 0.1036 * x ** 4)
    yU = yc + yt * np.cos(th)
    yL = yc - yt * np.cos(th)
    xe = np.zeros((2 * N - 1, 2))
    for i in range(N):
        xe[i] = [x[i] - x0, yU[i]]
    for i in range(N - 1):
        xe[i + N] = [x[N - 2 - i] - x0, yL[N - 2 - i]]
    xe *= chord
    if aoa != 0.0:
        c, s = math.cos(-aoa), math.sin(-aoa)
        X = xe[:, 0] - pivot[0]
        Y = xe[:, 1] - pivot[1]
        xe = np.stack([c * X - s * Y + pivot[0], s * X + c * Y + pivot[1]], axis=1)
    return RigidBody(xb=(xe[1:] + xe[:-1]) / 2.0, ds=np.sqrt(np.sum((xe[1:] - xe[:-1]) ** 2, axis=1)),
                     motion=motion)


# --------------------------------------------------------------------------
# Problem and state
# --------------------------------------------------------------------------
class IBProblem:
    """IBProblem(grid, bodies, dt, Re; freestream) on the GPU.

    ``freestream`` = (Ux, Uy, inclination): constants or callables of t,
    evaluated at t = 0 as the reference's IBState does for static bodies
    (state-types.jl:45, timestepping.jl:252-270).  The handle owns the device
    state; ``IBState`` objects are host mirrors of it.

    ``precision``: "fp64" (the reference's arithmetic) or "fp32_refined"
    (FP32 sine transforms in the projection solve and the final vort2flux!,
    each corrected by ``refine_sweeps`` sweeps of FP64-residual iterative
    refinement started from the previous solution; state, stencils, the
    trial solve and trial vort2flux!, Schur solve and forces FP64).

    A body whose ``motion`` is a ``MovingGrid`` (one body only, models.jl:137)
    makes every ``advance`` recompute the base flux from the motion at each
    step's t (timestepping.jl:41-43, 273-318); the free stream is then added
    to the motion's (the reference's default free stream is zero).  Bodies
    whose motions are all ``MotionFunction``s move every step, with E and B⁻¹
    rebuilt on the device (timestepping.jl:386-398).
    """

    def __init__(self, grid, bodies, dt, Re, freestream=(1.0, 0.0, 0.0), beta=(1.5, -0.5),
                 device=0, sync_fields=True, precision="fp64", refine_sweeps=1):
        self.lib = load_library()
        self.grid = grid
        self.bodies = list(bodies)
        self.dt = float(dt)
        self.Re = float(Re)
        ev = [f(0.0) if callable(f) else float(f) for f in freestream]
        self.freestream = tuple(ev)
        self.sync_fields = sync_fields
        xb = np.concatenate([b.xb for b in self.bodies], axis=0)
        self.nb = xb.shape[0]
        self.nf = 2 * self.nb
        self._xb = np.ascontiguousarray(xb.T.reshape(-1))      # column-major (nb, 2)
        self._ds = np.ascontiguousarray(np.concatenate([b.ds for b in self.bodies]).astype(np.float64))
        self._npts = (C.c_int32 * len(self.bodies))(*[b.xb.shape[0] for b in self.bodies])
        d = self._desc_of(grid, ev, beta, precision, device, refine_sweeps)
        h = C.c_void_p()
        rc = self.lib.ibpm_create(C.byref(d), C.byref(h))
        if rc != IBPM_OK:
            raise IBPMError(rc, self.lib.ibpm_last_error(None).decode())
        self.handle = h
        self._owns = True
        moving = [b.motion for b in self.bodies if isinstance(b.motion, MovingGrid)]
        self.motion = moving[0] if moving else None
        mfs = [b.motion for b in self.bodies if isinstance(b.motion, MotionFunction)]
        self.body_motions = None
        if mfs:
            if len(mfs) != len(self.bodies) or self.motion is not None:
                self.close()
                raise IBPMError(IBPM_ERR_UNSUPPORTED, "either every body has a MotionFunction or none")
            self.body_motions = mfs
            self._check(self.lib.ibpm_set_motion_function(self.handle))
        if self.motion is not None:
            if len(self.bodies) != 1:
                self.close()
                raise IBPMError(IBPM_ERR_UNSUPPORTED, "a moving grid carries exactly one body")
            m0 = np.array(self.motion.row(0.0))
            self._check(self.lib.ibpm_set_moving_grid(self.handle, 0.0, 0.0, _ptr(m0)))

    def _desc_of(self, grid, ev, beta, precision, device, refine_sweeps):
        d = ProblemDesc()
        d.nx, d.ny, d.mg = grid.nx, grid.ny, grid.mg
        d.h, d.offx, d.offy = grid.h, grid.offx, grid.offy
        d.Re, d.dt = self.Re, self.dt
        d.Ux, d.Uy, d.inclination = ev
        d.beta[0], d.beta[1] = beta
        d.nbodies, d.nb = len(self.bodies), self.nb
        d.body_npts = C.cast(self._npts, C.POINTER(C.c_int32))
        d.xb = self._xb.ctypes.data_as(_DP)
        d.ds = self._ds.ctypes.data_as(_DP)
        if precision not in PRECISIONS:
            raise IBPMError(IBPM_ERR_INVALID, "precision must be one of %s" % sorted(PRECISIONS))
        self.precision = precision
        d.precision = PRECISIONS[precision]
        d.device = device
        d.refine_sweeps = int(refine_sweeps)
        self._desc = d
        return d

    def _check(self, rc):
        if rc != IBPM_OK:
            raise IBPMError(rc, self.lib.ibpm_last_error(self.handle).decode())

    def close(self):
        if getattr(self, "handle", None):
            if getattr(self, "_owns", True):
                self.lib.ibpm_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_base_state(self, base):
        """LinearizedIBProblem(base, prob, dt) (problem-types.jl:47-87): step the
        linearisation about the host state ``base`` (its Γ and q; the base flux
        is the problem's) from now on.  The state's own q0 becomes zero."""
        G = np.asfortranarray(base.Gamma, dtype=np.float64)
        q = np.asfortranarray(base.q, dtype=np.float64)
        self._check(self.lib.ibpm_set_base_state(self.handle, _ptr(G), _ptr(q)))

    def binv(self):
        """prob.Binv (laplacian.jl:118) as an (nf, nf) array."""
        out = np.empty((self.nf, self.nf), order="F")
        self._check(self.lib.ibpm_get_binv(self.handle, out.ctypes.data_as(_DP)))
        return out

    def sync(self):
        self._check(self.lib.ibpm_sync(self.handle))


class IBState:
    """Host mirror of IBState (state-types.jl:7-22): q, q0 (nq, mg); Γ, ψ,
    nonlin[k] (nΓ, mg); F̃b (nf, 1); CD, CL per body — all column-major."""

    def __init__(self, prob):
        g = prob.grid
        self.q = np.zeros((g.nq, g.mg), order="F")
        self.q0 = np.zeros((g.nq, g.mg), order="F")
        self.Gamma = np.zeros((g.nGamma, g.mg), order="F")
        self.psi = np.zeros((g.nGamma, g.mg), order="F")
        self.nonlin = [np.zeros((g.nGamma, g.mg), order="F"), np.zeros((g.nGamma, g.mg), order="F")]
        self.Fb = np.zeros((prob.nf, 1), order="F")
        self.CD = np.zeros(len(prob.bodies))
        self.CL = np.zeros(len(prob.bodies))
        pull_state(self, prob)

    # The vector space of states (state-types.jl:57-155): scaling and sums act
    # on Γ, q, ψ and the nonlinear terms; the inner product is that of q (the
    # kinetic energy), as Krylov stability runs use it
    # (benchmarks/cyl40_stability/run_krylov.jl:30-42).
    _VEC = ("Gamma", "q", "psi")

    def copy(self):
        """copy!(similar(v), v): a host mirror with every field copied."""
        w = IBState.__new__(IBState)
        for name in ("q", "q0", "Gamma", "psi", "Fb", "CD", "CL"):
            setattr(w, name, np.array(getattr(self, name), order="F"))
        w.nonlin = [np.array(a, order="F") for a in self.nonlin]
        return w

    def rmul(self, alpha):
        """rmul!(v, α): v ← α v in place."""
        for name in self._VEC:
            getattr(self, name)[...] *= alpha
        for a in self.nonlin:
            a *= alpha
        return self

    def axpby(self, alpha, v, beta):
        """axpby!(α, v, β, w) with w = self: w ← α v + β w, evaluated as the
        reference does, (β/α w + v) α."""
        self.rmul(beta / alpha)
        for name in self._VEC:
            getattr(self, name)[...] += getattr(v, name)
        for a, b in zip(self.nonlin, v.nonlin):
            a += b
        return self.rmul(alpha)

    def axpy(self, alpha, v):
        """axpy!(α, v, w) with w = self: w ← α v + w."""
        return self.axpby(alpha, v, 1.0)

    def dot(self, other):
        """dot(v, w) = dot(v.q, w.q)."""
        return float(np.vdot(self.q, other.q))

    def norm(self):
        """norm(v) = norm(v.q)."""
        return float(np.linalg.norm(self.q))


class PinnedArray:
    """A float64 numpy array over page-locked host memory from ibpm_host_alloc."""

    def __init__(self, shape, order="F"):
        lib = load_library()
        n = int(np.prod(shape))
        self._lib = lib
        self._p = lib.ibpm_host_alloc(8 * max(n, 1))
        if not self._p:
            raise IBPMError(IBPM_ERR_NOMEM, "ibpm_host_alloc failed")
        buf = (C.c_double * max(n, 1)).from_address(self._p)
        self.array = np.ndarray(shape, dtype=np.float64, buffer=buf, order=order)
        self.array[...] = 0.0

    def free(self):
        if self._p:
            self.array = None
            self._lib.ibpm_host_free(self._p)
            self._p = None


def pinned_state(prob):
    """An IBState whose arrays live in page-locked host memory."""
    g = prob.grid
    keep = []

    def mk(shape):
        pa = PinnedArray(shape)
        keep.append(pa)
        return pa.array

    st = IBState.__new__(IBState)
    st.q, st.q0 = mk((g.nq, g.mg)), mk((g.nq, g.mg))
    st.Gamma, st.psi = mk((g.nGamma, g.mg)), mk((g.nGamma, g.mg))
    st.nonlin = [mk((g.nGamma, g.mg)), mk((g.nGamma, g.mg))]
    st.Fb = mk((prob.nf, 1))
    st.CD = np.zeros(len(prob.bodies))
    st.CL = np.zeros(len(prob.bodies))
    st._pinned = keep
    pull_state(st, prob)
    return st


def kernel_names():
    lib = load_library()
    return [lib.ibpm_kernel_name(k).decode() for k in range(KERNEL_COUNT)]


def bench_steps(prob, nsteps, flush_l2=True):
    """Per-step device times (ms) of nsteps graph replays (ibpm_bench)."""
    out = np.zeros(nsteps)
    prob._check(prob.lib.ibpm_bench(prob.handle, int(nsteps), int(bool(flush_l2)), out.ctypes.data_as(_DP)))
    return out


def profile_steps(prob, nsteps, flush_l2=True):
    """Per-kernel-class (ms, algorithmic bytes, launches) over nsteps eager steps."""
    ms = np.zeros(KERNEL_COUNT)
    by = np.zeros(KERNEL_COUNT)
    calls = np.zeros(KERNEL_COUNT, dtype=np.int32)
    prob._check(prob.lib.ibpm_profile(prob.handle, int(nsteps), int(bool(flush_l2)), ms.ctypes.data_as(_DP),
                                      by.ctypes.data_as(_DP), calls.ctypes.data_as(C.POINTER(C.c_int32))))
    return {n: (ms[k], by[k], int(calls[k])) for k, n in enumerate(kernel_names())}


def launches_per_step(prob):
    n = prob.lib.ibpm_launches_per_step(prob.handle)
    if n < 0:
        prob._check(n)
    return n


def set_transform_plan(prob, single_slab=IBPM_PLAN_LATENCY, multi_slab=IBPM_PLAN_AUTO):
    """Plans of the problem's sine transforms, for launches over one level
    (IBPM_PLAN_LATENCY or IBPM_PLAN_THROUGHPUT) and over several (either, or
    IBPM_PLAN_AUTO: the throughput plan from 4 slabs on)."""
    prob._check(prob.lib.ibpm_set_transform_plan(prob.handle, int(single_slab), int(multi_slab)))


def transform_plan(prob):
    """(single-slab plan, multi-slab plan) of the problem."""
    a, b = C.c_int32(), C.c_int32()
    prob._check(prob.lib.ibpm_get_transform_plan(prob.handle, C.byref(a), C.byref(b)))
    return a.value, b.value


def set_level_chain(prob, chain):
    """How vort2flux! runs its levels: IBPM_CHAIN_SEQUENTIAL (the reference's
    order) or IBPM_CHAIN_BOUNDARY_TRANSFER (the default where its factors
    exist).  The results agree to rounding."""
    prob._check(prob.lib.ibpm_set_level_chain(prob.handle, int(chain)))


def level_chain(prob):
    """The problem's level chain (IBPM_CHAIN_*)."""
    c = C.c_int32()
    prob._check(prob.lib.ibpm_get_level_chain(prob.handle, C.byref(c)))
    return c.value


def _field_shapes(prob):
    g = prob.grid
    return {"Gamma": (g.nGamma, g.mg), "q": (g.nq, g.mg), "q0": (g.nq, g.mg), "psi": (g.nGamma, g.mg),
            "nonlin": (g.nGamma, g.mg), "Fb": (prob.nf, 1)}


def _checked(prob, name, a, writable=False):
    """``a`` as the library reads or writes it: float64, column-major, of the
    field's shape.  A wrong shape raises (the C ABI takes bare pointers and
    cannot tell)."""
    shape = _field_shapes(prob)[name]
    a = np.asarray(a)
    if a.ndim == 1 and shape[1] == 1:
        a = a.reshape(shape, order="F")
    if a.shape != shape:
        raise IBPMError(IBPM_ERR_INVALID, "state.%s must have shape %s, not %s" % (name, shape, a.shape))
    if writable and not (a.dtype == np.float64 and a.flags.f_contiguous and a.flags.writeable):
        raise IBPMError(IBPM_ERR_INVALID, "state.%s must be a writable column-major float64 array" % name)
    return a if writable else np.asfortranarray(a, dtype=np.float64)


def pull_state(state, prob):
    """Copy the device state into ``state``."""
    dst = [_checked(prob, "Gamma", state.Gamma, True), _checked(prob, "q", state.q, True),
           _checked(prob, "q0", state.q0, True), _checked(prob, "psi", state.psi, True),
           _checked(prob, "nonlin", state.nonlin[0], True), _checked(prob, "nonlin", state.nonlin[1], True),
           _checked(prob, "Fb", state.Fb, True)]
    prob._check(prob.lib.ibpm_get_state(prob.handle, *[_ptr(a) for a in dst]))


def push_state(state, prob, fields=("Gamma", "q", "q0", "psi", "nonlin", "Fb")):
    """Copy ``state`` (the listed fields) to the device."""
    f = set(fields)

    def arr(name, a):
        return _checked(prob, name, a) if name in f else None

    keep = [arr("Gamma", state.Gamma), arr("q", state.q), arr("q0", state.q0), arr("psi", state.psi),
            arr("nonlin", state.nonlin[0]), arr("nonlin", state.nonlin[1]), arr("Fb", state.Fb)]
    prob._check(prob.lib.ibpm_set_state(prob.handle, *[_ptr(a) for a in keep]))


def advance(state, prob, t=0.0, nsteps=1):
    """advance!(state, prob, t) — ``nsteps`` steps on the device at times
    t, t + dt, … (or at the times of ``t`` when it is an array).  Returns the
    (nsteps, nbodies) CD and CL histories; state.CD/CL hold the last row.
    Fields are copied back when ``prob.sync_fields`` is set."""
    nbod = len(prob.bodies)
    ts = np.atleast_1d(np.asarray(t, dtype=np.float64))
    if ts.size > 1 or np.ndim(t) == 1:
        nsteps = ts.size
    cd = np.zeros((nsteps, nbod))
    cl = np.zeros((nsteps, nbod))
    if getattr(prob, "body_motions", None):
        if ts.size != nsteps:
            ts = ts[0] + prob.dt * np.arange(nsteps)
        rows = np.ascontiguousarray([[m.row(tk) for m in prob.body_motions] for tk in ts],
                                    dtype=np.float64).reshape(-1)
        rc = prob.lib.ibpm_advance_bodies(prob.handle, int(nsteps), _ptr(rows), cd.ctypes.data_as(_DP),
                                          cl.ctypes.data_as(_DP))
    elif getattr(prob, "motion", None) is not None:
        if ts.size != nsteps:
            ts = ts[0] + prob.dt * np.arange(nsteps)
        rows = np.ascontiguousarray([prob.motion.row(tk) for tk in ts], dtype=np.float64).reshape(-1)
        rc = prob.lib.ibpm_advance_moving(prob.handle, int(nsteps), _ptr(rows), cd.ctypes.data_as(_DP),
                                          cl.ctypes.data_as(_DP))
    else:
        rc = prob.lib.ibpm_advance(prob.handle, float(ts[0]) if ts.size else 0.0, int(nsteps),
                                   cd.ctypes.data_as(_DP), cl.ctypes.data_as(_DP))
    if nsteps:
        state.CD[:] = cd[-1]
        state.CL[:] = cl[-1]
    if prob.sync_fields:
        pull_state(state, prob)
    if rc != IBPM_OK:
        err = IBPMError(rc, prob.lib.ibpm_last_error(prob.handle).decode())
        err.CD, err.CL = cd, cl     # the histories up to the failure (non-finite rows included)
        raise err
    return cd, cl


def body_points(prob):
    """The body points and their velocities after the last step (state.xb and
    the bodies' ub), each (nb, 2)."""
    xb = np.zeros((prob.nb, 2), order="F")
    ub = np.zeros((prob.nb, 2), order="F")
    prob._check(prob.lib.ibpm_get_body_points(prob.handle, _ptr(xb), _ptr(ub)))
    return xb, ub


def vort2flux(state, prob):
    """vort2flux!(state.ψ, state.q, state.Γ, model, mg) on the device state."""
    prob._check(prob.lib.ibpm_vort2flux(prob.handle))
    pull_state(state, prob)


def run_sim(t, state, prob):
    """run_sim! of src/ibpm.jl:90-106 without logging: one step per entry of
    ``t``.  Like the reference (src/ibpm.jl:95-97) it stops quietly at the
    first step whose lift coefficient is not finite: the histories returned
    end with that step's row."""
    try:
        return advance(state, prob, np.asarray(t, dtype=np.float64), nsteps=len(t))
    except IBPMError as e:
        if e.code != IBPM_ERR_NONFINITE:
            raise
        bad = np.flatnonzero(~np.all(np.isfinite(e.CL), axis=1))
        last = int(bad[0]) + 1 if bad.size else len(e.CL)
        return e.CD[:last], e.CL[:last]


# --------------------------------------------------------------------------
# Discrete adjoint
# --------------------------------------------------------------------------
@dataclass
class AdjointResult:
    J: float
    grad_Gamma0: np.ndarray     # (nΓ, mg), like state.Gamma
    grad_q0: np.ndarray         # (nq, mg), like state.q
    grad_omega0: np.ndarray     # (nΓ,): for a start state built from a finest-level vorticity
    grad_alpha: float           # freestream angle
    grad_xb: np.ndarray = None  # (nb, 2): body-point positions (when asked for)


def adjoint_run(prob, nsteps, k_checkpoint=50, window=None, w_cd=1.0, w_cl=0.0, want_xb=False):
    """Gradient of J = mean over the last ``window`` steps of Σ_bodies
    (w_cd·CD + w_cl·CL) over ``nsteps`` steps of advance! from the problem's
    current device state, by the discrete adjoint with a checkpoint every
    ``k_checkpoint`` steps; with ``want_xb`` also with respect to the
    body-point positions.  The device state ends at the final state of the
    run (pull it with ``pull_state``)."""
    lib = prob.lib
    window = nsteps if window is None else window
    obj = Objective(window=int(window), w_cd=float(w_cd), w_cl=float(w_cl))
    nG, nq, mg = prob.grid.nGamma, prob.grid.nq, prob.grid.mg
    J = C.c_double()
    gG = np.zeros((nG, mg), order="F")
    gq = np.zeros((nq, mg), order="F")
    gw = np.zeros(nG)
    ga = C.c_double()
    gx = np.zeros((prob.nb, 2), order="F") if want_xb else None
    prob._check(lib.ibpm_adjoint_run(prob.handle, int(nsteps), int(k_checkpoint), C.byref(obj), C.byref(J),
                                     _ptr(gG), _ptr(gq), _ptr(gw), C.byref(ga), _ptr(gx)))
    return AdjointResult(J=J.value, grad_Gamma0=gG, grad_q0=gq, grad_omega0=gw, grad_alpha=ga.value, grad_xb=gx)


def adjoint_bench_steps(prob, nsteps, flush_l2=True):
    """Device ms of the adjoint of one step, ``nsteps`` replays (after an
    ``adjoint_run`` on the problem)."""
    out = np.zeros(nsteps)
    prob._check(prob.lib.ibpm_adjoint_bench(prob.handle, int(nsteps), 1 if flush_l2 else 0, _ptr(out)))
    return out


# --------------------------------------------------------------------------
# Batches of independent simulations
# --------------------------------------------------------------------------
class Batch:
    """Many independent simulations advanced together: one CUDA-graph launch
    per step whose branches are the members' steps over ``lanes`` concurrent
    streams (``lanes=0`` picks the count by timing).  ``members`` are
    IBProblem-like objects for push_state / pull_state / vort2flux; step them
    only through the batch.  ``specs`` is a list of dicts with the IBProblem
    arguments (grid, bodies, dt, Re and optionally freestream, beta,
    precision, refine_sweeps)."""

    def __init__(self, specs, lanes=0, device=0):
        self.lib = load_library()
        self.members = []
        descs = (ProblemDesc * len(specs))()
        keep = []
        for i, sp_ in enumerate(specs):
            m = IBProblem.__new__(IBProblem)
            m.lib = self.lib
            m.grid = sp_["grid"]
            m.bodies = list(sp_["bodies"])
            if any(b.motion is not None for b in m.bodies):
                raise IBPMError(IBPM_ERR_UNSUPPORTED, "member %d: moving bodies or grids are not batched" % i)
            m.motion = None
            m.body_motions = None
            m.dt = float(sp_["dt"])
            m.Re = float(sp_["Re"])
            fs = sp_.get("freestream", (1.0, 0.0, 0.0))
            ev = tuple(f(0.0) if callable(f) else float(f) for f in fs)
            m.freestream = ev
            m.sync_fields = sp_.get("sync_fields", False)
            xb = np.concatenate([b.xb for b in m.bodies], axis=0)
            m.nb = xb.shape[0]
            m.nf = 2 * m.nb
            m._xb = np.ascontiguousarray(xb.T.reshape(-1))
            m._ds = np.ascontiguousarray(np.concatenate([b.ds for b in m.bodies]).astype(np.float64))
            m._npts = (C.c_int32 * len(m.bodies))(*[b.xb.shape[0] for b in m.bodies])
            m.Re = float(sp_["Re"])
            d = m._desc_of(m.grid, ev, sp_.get("beta", (1.5, -0.5)), sp_.get("precision", "fp64"), device,
                           sp_.get("refine_sweeps", 1))
            descs[i] = d
            keep.append(m)
            self.members.append(m)
        h = C.c_void_p()
        rc = self.lib.ibpm_batch_create(len(specs), descs, int(lanes), C.byref(h))
        if rc != IBPM_OK:
            raise IBPMError(rc, self.lib.ibpm_batch_last_error(None).decode())
        self.handle = h
        for i, m in enumerate(self.members):
            m.handle = C.c_void_p(self.lib.ibpm_batch_member(h, i))
            m._owns = False

    def _check(self, rc):
        if rc != IBPM_OK:
            raise IBPMError(rc, self.lib.ibpm_batch_last_error(self.handle).decode())

    @property
    def lanes(self):
        return self.lib.ibpm_batch_lanes(self.handle)

    def set_lanes(self, lanes):
        self._check(self.lib.ibpm_batch_set_lanes(self.handle, int(lanes)))

    @property
    def plan(self):
        """Transform plan of the members' single-level launches."""
        return self.lib.ibpm_batch_plan(self.handle)

    def set_plan(self, plan):
        self._check(self.lib.ibpm_batch_set_plan(self.handle, int(plan)))

    @property
    def chain(self):
        """Level chain of the members' vort2flux! (IBPM_CHAIN_*)."""
        return self.lib.ibpm_batch_chain(self.handle)

    def set_chain(self, chain):
        self._check(self.lib.ibpm_batch_set_chain(self.handle, int(chain)))

    @property
    def grouped(self):
        """Whether members of one grid and precision step by shared launches."""
        return bool(self.lib.ibpm_batch_grouped(self.handle))

    def set_grouped(self, on):
        self._check(self.lib.ibpm_batch_set_grouped(self.handle, 1 if on else 0))

    def advance(self, nsteps=1):
        """Advance every member; returns per-member (CD, CL) histories (nsteps, nbodies)."""
        self._check(self.lib.ibpm_batch_advance(self.handle, int(nsteps)))
        out = []
        for i, m in enumerate(self.members):
            cd = np.zeros((nsteps, len(m.bodies)))
            cl = np.zeros((nsteps, len(m.bodies)))
            self._check(self.lib.ibpm_batch_get_forces(self.handle, i, _ptr(cd), _ptr(cl)))
            out.append((cd, cl))
        return out

    def bench_steps(self, nsteps, flush_l2=True):
        out = np.zeros(nsteps)
        self._check(self.lib.ibpm_batch_bench(self.handle, int(nsteps), 1 if flush_l2 else 0, _ptr(out)))
        return out

    def close(self):
        if getattr(self, "handle", None):
            for m in self.members:
                m.handle = None
            self.lib.ibpm_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
