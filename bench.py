#!/usr/bin/env python
"""Benchmark of the IBPM time step (advance!) on B200.

Workload: a circular cylinder, D = 1 at the origin, with
314 boundary points (≈ 1 point per h), at Re = 100 in a uniform freestream
U = 1 along x; 512×512 cells per level, h = 0.01 (finest domain
x ∈ [-1, 4.12], y ∈ [-2.56, 2.56]), 5 nested levels, dt = 0.002.  The start
state is a Gaussian vortex perturbation ω = 1e-3 exp(-r²/0.2²) centred at
(1.5, 0.1) on the finest level (Γ = h² ω, then vort2flux!).  All inputs are
synthetic; nothing is read from a dataset.

Our arm (default): one process per GPU (torchrun for N > 1, replicas of the
same simulation: one simulation does not shard, every 2-D sine transform
couples a whole level), K steps replayed from a CUDA graph, each timed by CUDA
events on the library's stream with a 512 MiB L2 flush between steps (outside
the timed pairs).  value = Σ_ranks nx·ny·mg·K / max_ranks(Σ step times) of the
FP32-refined path; the plain FP64 path is timed the same way beside it, with
the CD/CL differences between the two over the same K steps.

--impl reference: the FP64 CPU restatement of the reference's step
(oracle/ibpm_ref.py, numpy + scipy.fft with all host threads) on the same
workload, rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "ibpm.jl_b200", "python"))

# The workload: 512x512 cells x 5 levels, h = 0.01, Re = 100, dt = 0.002.
H = 0.01
BOUNDARY = (-1.0, 4.12, -2.56, 2.56)
MG = 5
RE = 100.0
DT = 0.002
NB = 314
VORTEX = dict(amp=1e-3, width=0.2, x0=1.5, y0=0.1)
WORKLOAD = ("cylinder D=1 (314 pts) Re=100, 512x512 cells x 5 levels, h=0.01, dt=0.002, "
            "Gaussian-vortex start (1e-3, 0.2, (1.5, 0.1))")
METRIC = "cell-steps/s"
FALLBACK_HBM_GBS = 6650.0
REF_MAX_STEPS = 100

# Algorithmic bytes of one FP64 step: s·nΓ·(34.5·mg + 3.5) + 8·nf² with s = 8
# (every operator reads its inputs once and writes its outputs once; each 2-D
# DST-I one read + one write of nΓ; 8·mg+2 DSTs per step).
def step_bytes_model(nx, ny, mg, nf, s=8):
    nG = (nx - 1) * (ny - 1)
    return s * nG * (34.5 * mg + 3.5) + 8 * nf * nf


def vortex_gamma(nx, ny, mg, h, offx, offy):
    """Γ (nΓ, mg) column-major: h²·ω at the finest-level vertices, 0 elsewhere."""
    i = np.arange(1, nx)
    j = np.arange(1, ny)
    X = i[:, None] * h - offx
    Y = j[None, :] * h - offy
    r2 = (X - VORTEX["x0"]) ** 2 + (Y - VORTEX["y0"]) ** 2
    w = VORTEX["amp"] * np.exp(-r2 / VORTEX["width"] ** 2)
    G = np.zeros(((nx - 1) * (ny - 1), mg), order="F")
    G[:, 0] = (h * h * w).flatten(order="F")
    return G


def read_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def read_traffic(kernel):
    """DRAM bytes per launch of `kernel` from a committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        d = json.load(open(p))
        return d.get(kernel)
    except Exception:
        return None


# --------------------------------------------------------------------------
# Clock sampling (nvidia-smi, during the timed region)
# --------------------------------------------------------------------------
SMI_Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")


class ClockSampler:
    def __init__(self, device):
        self.device = device
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + SMI_Q,
                                       "--format=csv,noheader,nounits", "-lms", "100"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None
        time.sleep(0.3)

    def stop(self):
        if self.p is None:
            return None
        time.sleep(0.15)
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        rows = [r.split(",") for r in open(self.f.name).read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [x.strip() for x in r]
            if len(r) < 9:
                continue
            try:
                sm.append(float(r[1]))
                mx.append(float(r[2]))
            except ValueError:
                continue
            for n, v in zip(names, r[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


# --------------------------------------------------------------------------
# Distributed plumbing (replicas; barrier and max only)
# --------------------------------------------------------------------------
def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


class Dist:
    def __init__(self):
        self.world, self.rank, self.local = dist_env()
        self.pg = None
        if self.world > 1:
            import datetime

            import torch.distributed as dist
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=300))
            self.dist = dist

    def barrier(self):
        if self.world > 1:
            self.dist.barrier()

    def max(self, x):
        if self.world == 1:
            return x
        import torch
        t = torch.tensor([float(x)], dtype=torch.float64)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.world > 1:
            self.dist.destroy_process_group()


# --------------------------------------------------------------------------
# CPU arms (oracle)
# --------------------------------------------------------------------------
def cpu_problem(threads):
    from oracle import ibpm_ref as R
    R.WORKERS = threads
    g = R.make_grid(H, BOUNDARY, MG)
    p = R.IBProblem(grid=g, bodies=[R.make_cylinder(0.5, g.h, 0.0, 0.0, n=NB)], dt=DT, Re=RE,
                    build_binv=False)
    # The dense Schur solve costs one nf×nf GEMV per step whatever the matrix;
    # a seeded dense matrix of the right size stands in for B⁻¹ in timing runs.
    p.Binv = np.random.default_rng(0).standard_normal((p.nf, p.nf)) * 1e-3
    st = R.make_state(p)
    st.Gamma = np.stack([R.gamma_from_ref(vortex_gamma(g.nx, g.ny, g.mg, g.h, g.offx, g.offy), g)[l]
                         for l in range(g.mg)])
    R.refresh_flux(st, p)
    return R, g, p, st


def cpu_step_rate(steps, threads):
    R, g, p, st = cpu_problem(threads)
    R.advance(st, p)  # warm-up
    t0 = time.perf_counter()
    for _ in range(steps):
        R.advance(st, p)
    dt = time.perf_counter() - t0
    return g.nx * g.ny * g.mg * steps / dt, dt


def run_reference(args, d):
    if d.rank != 0:
        return 0
    threads = os.cpu_count() or 1
    R, g, p, st = cpu_problem(threads)
    # bounded sample: at most REF_MAX_STEPS timed steps (≈ 0.2 s each on 8 cores)
    nsteps = min(args.steps, REF_MAX_STEPS)
    nwarm = min(args.warmup, 3)
    for _ in range(nwarm):
        R.advance(st, p)
    t0 = time.perf_counter()
    for _ in range(nsteps):
        R.advance(st, p)
    wall = time.perf_counter() - t0
    value = g.nx * g.ny * g.mg * nsteps / wall
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": args.gpus,
        "steps": nsteps, "warmup": nwarm, "ms_per_step": 1e3 * wall / nsteps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": WORKLOAD, "precision": "fp64", "implementation":
                   "oracle/ibpm_ref.py: FP64 numpy/scipy restatement of the reference's advance! "
                   "(the Julia reference itself cannot run here: no Julia toolchain)"},
        "cpu_baseline": {"value": value, "unit": METRIC, "cores": threads, "kind": "port",
                         "sample": "%d steps of the workload after %d warm-up steps (requested %d, capped "
                                   "at %d); B^-1 replaced by a seeded dense matrix of the same size"
                                   % (nsteps, nwarm, args.steps, REF_MAX_STEPS)},
        "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


# --------------------------------------------------------------------------
# Our arm
# --------------------------------------------------------------------------
def measure(args, d, precision, sampler=None):
    """Time one precision mode on the workload: K graph replays (device-timed,
    L2 flushed between steps), then K advance! calls through the public API
    with host buffers (e2e, CD/CL history kept), then a per-kernel profile."""
    import ibpm_gpu as G
    dev = d.local
    g = G.make_grid(H, BOUNDARY, MG)
    body = G.make_cylinder(0.5, g.h, 0.0, 0.0, n=NB)
    prob = G.IBProblem(g, [body], DT, RE, freestream=(1.0, 0.0, 0.0), device=dev, sync_fields=False,
                       precision=precision, refine_sweeps=1)
    cells = g.nx * g.ny * g.mg

    # seeded start state through the public API (pinned host mirror)
    st = G.pinned_state(prob)
    st.Gamma[...] = vortex_gamma(g.nx, g.ny, g.mg, g.h, g.offx, g.offy)
    G.push_state(st, prob, fields=("Gamma",))
    G.vort2flux(st, prob)
    init = {k: np.array(getattr(st, k)) for k in ("Gamma", "q", "q0", "psi")}
    init_nl = [np.array(a) for a in st.nonlin]

    # graph capture + first replays; the 32 start-up steps of the
    # FP32-refined path (two correction sweeps each) fall in the warm-up, so
    # the K timed steps are those of a long run
    G.bench_steps(prob, max(args.warmup, 40), flush_l2=True)

    d.barrier()
    if sampler:
        sampler.start()
    step_ms = G.bench_steps(prob, args.steps, flush_l2=True)
    clocks = sampler.stop() if sampler else None
    total_ms = d.max(float(np.sum(step_ms)))

    # end to end: upload the state from pinned memory, K advance! calls (each
    # returns CD/CL to the host), download the state
    for k, v in init.items():
        getattr(st, k)[...] = v
    st.nonlin[0][...] = init_nl[0]
    st.nonlin[1][...] = init_nl[1]
    prob.sync()
    cd = np.zeros(args.steps)
    cl = np.zeros(args.steps)
    d.barrier()
    t0 = time.perf_counter()
    G.push_state(st, prob)
    for k in range(args.steps):
        c, l = G.advance(st, prob, k * DT, nsteps=1)
        cd[k], cl[k] = c[0, 0], l[0, 0]
    G.pull_state(st, prob)
    e2e_s = d.max(time.perf_counter() - t0)
    state_bytes = 8 * (st.Gamma.size * 4 + st.q.size * 2 + st.Fb.size)
    gamma = np.array(st.Gamma)

    prof = G.profile_steps(prob, 4, flush_l2=True)
    lps = G.launches_per_step(prob)
    nf = prob.nf
    prob.close()
    return dict(cells=cells, nf=nf, g=g, total_ms=total_ms, e2e_s=e2e_s, cd=cd, cl=cl, prof=prof, lps=lps,
                clocks=clocks, state_bytes=state_bytes, bodies=1, gamma=gamma)


# The adjoint workload: a cylinder at Re = 100 on 256x256 cells x 4 levels
# (h = 0.02, same domain), dt = 0.004, 1000 steps; J = the drag averaged over
# the last 200 steps; start state from a seeded N(0, (1e-4)²) vorticity per
# finest cell; a checkpoint every 50 steps.
ADJ = dict(h=0.02, mg=4, dt=0.004, nb=157, steps=1000, window=200, k=50, sigma=1e-4, seed=11)
ADJ_WORKLOAD = ("adjoint of mean drag (last 200 of 1000 steps), cylinder D=1 (157 pts) Re=100, 256x256 cells "
                "x 4 levels, h=0.02, dt=0.004, N(0,1e-4) start vorticity, checkpoint every 50 steps")


def measure_adjoint(args, d, precision="fp64"):
    """Wall time of ibpm_adjoint_run (forward with checkpoints, recomputation,
    adjoint sweep) against ibpm_advance over the same steps, the device time
    of one adjoint step against one forward step, and a central-difference
    check of ⟨∂J/∂ω, d⟩ (ε = 1e-6) through two forward runs."""
    import ibpm_gpu as G
    g = G.make_grid(ADJ["h"], BOUNDARY, ADJ["mg"])
    body = G.make_cylinder(0.5, g.h, 0.0, 0.0, n=ADJ["nb"])
    prob = G.IBProblem(g, [body], ADJ["dt"], RE, device=d.local, sync_fields=False, precision=precision)
    rng = np.random.default_rng(ADJ["seed"])
    w0 = ADJ["sigma"] * rng.standard_normal((g.nx - 1, g.ny - 1))
    dirn = rng.standard_normal(w0.shape)
    st = G.IBState(prob)
    n = ADJ["steps"]

    def start(w):
        for a in (st.Gamma, st.q, st.psi, st.nonlin[0], st.nonlin[1], st.Fb):
            a[...] = 0.0
        st.Gamma[:, 0] = g.h ** 2 * w.flatten(order="F")
        G.push_state(st, prob)
        G.vort2flux(st, prob)

    def forward(w):
        start(w)
        prob.sync()
        t0 = time.perf_counter()
        cd, _ = G.advance(st, prob, 0.0, nsteps=n)
        return time.perf_counter() - t0, float(np.mean(cd[-ADJ["window"]:, 0]))

    forward(w0)                                   # warm-up (graph capture)
    start(w0)
    G.adjoint_run(prob, n, ADJ["k"], ADJ["window"])
    t_fwd, J0 = forward(w0)
    start(w0)
    prob.sync()
    t0 = time.perf_counter()
    res = G.adjoint_run(prob, n, ADJ["k"], ADJ["window"])
    t_adj = time.perf_counter() - t0
    eps = 1e-6
    _, Jp = forward(w0 + eps * dirn)
    _, Jm = forward(w0 - eps * dirn)
    fd = (Jp - Jm) / (2 * eps)
    ad = float(np.dot(res.grad_omega0.flatten(order="F"), dirn.flatten(order="F")))
    fwd_ms = float(np.mean(G.bench_steps(prob, 100, flush_l2=True)[10:]))
    adj_ms = float(np.mean(G.adjoint_bench_steps(prob, 100, flush_l2=True)[10:]))
    prob.close()
    return dict(J=res.J, J_forward=J0, grad_alpha=res.grad_alpha, grad_omega0=res.grad_omega0,
                forward_s=t_fwd, adjoint_run_s=t_adj, fd=fd, ad=ad, fwd_step_ms=fwd_ms, adj_step_ms=adj_ms)


# Position gradient: two cylinders (D = 1, 157 points each, centres (0, ±0.75))
# at Re = 150 on 256x256 cells x 4 levels (h = 0.02, same domain), dt = 0.004,
# 400 steps; J = the total lift averaged over the last 100 steps; ∂J/∂xb for
# all 314 boundary points; a checkpoint every 100 steps; checked by central
# differences (ε = 1e-5 h) along 8 seeded perturbations of all points.  The
# bodies sit (1.234e-2, -7.11e-3) off the stated centres: with a point on a
# grid line, grid samples fall exactly where the reference's smoothed delta has
# its ~1e-9 coefficient jumps (|r| = h, 2h, 3h), which differences would see.
XB = dict(h=0.02, mg=4, dt=0.004, nb=157, Re=150.0, steps=400, window=100, k=100, seed=7, ndir=8,
          off=(0.01234, -0.00711))
XB_WORKLOAD = ("position gradient of mean total lift (last 100 of 400 steps), two cylinders D=1 (157 pts each) at "
               "(0,+-0.75) Re=150, 256x256 cells x 4 levels, h=0.02, dt=0.004, checkpoint every 100 steps, "
               "8 seeded finite-difference directions")


# The large two-body workload: two cylinders D = 1 (628 points each) at
# (0, ±0.75), Re = 150, 1024x1024 cells x 5 levels, h = 0.005, dt = 0.001
# (nf = 2512), FP32-refined.  The block times `steps` steps of both paths from
# rest and their CD/CL differences, and the position gradient of the mean
# total lift (last 100 of `adj_steps` steps, checkpoint every 100) against
# finite differences along 8 seeded directions.
C5 = dict(h=0.005, mg=5, dt=0.001, nb=628, Re=150.0, steps=1000, hist_steps=10000, adj_steps=400, window=100, k=100,
          seed=7, ndir=8,
          off=(0.003085, -0.0017775))   # the gradient check moves the bodies off the grid lines (as XB, in h)
C5_WORKLOAD = ("two cylinders D=1 (628 pts each) at (0,+-0.75) Re=150, 1024x1024 cells x 5 levels, h=0.005, "
               "dt=0.001, nf=2512, from rest")


def c5_bodies(G, g, off=(0.0, 0.0), xb=None):
    ox, oy = off
    n = C5["nb"]
    bs = [G.make_cylinder(0.5, g.h, ox, 0.75 + oy, n=n), G.make_cylinder(0.5, g.h, ox, -0.75 + oy, n=n)]
    if xb is not None:
        bs[0].xb, bs[1].xb = xb[:n].copy(), xb[n:].copy()
    return bs


def config5_block(args, d):
    import ibpm_gpu as G
    g = G.make_grid(C5["h"], BOUNDARY, C5["mg"])
    cells = g.nx * g.ny * g.mg
    n, nh = C5["steps"], C5["hist_steps"]
    out = {"workload": C5_WORKLOAD, "metric": METRIC, "unit": METRIC}
    hist = {}
    for prec in ("fp32_refined", "fp64"):
        t0 = time.perf_counter()
        p = G.IBProblem(g, c5_bodies(G, g), C5["dt"], C5["Re"], device=d.local, sync_fields=False, precision=prec)
        setup_s = time.perf_counter() - t0
        st = G.IBState(p)
        G.bench_steps(p, 40, flush_l2=True)   # past the refined path's 32 two-sweep start-up steps
        ms = G.bench_steps(p, n, flush_l2=True)
        for a in (st.Gamma, st.q, st.psi, st.nonlin[0], st.nonlin[1], st.Fb):
            a[...] = 0.0
        G.push_state(st, p)
        p.sync()
        t0 = time.perf_counter()
        cd, cl = G.advance(st, p, 0.0, nsteps=nh)
        e2e_s = time.perf_counter() - t0
        hist[prec] = (cd, cl)
        out[prec] = {"value": cells * n / (float(np.sum(ms)) / 1e3), "ms_per_step": float(np.mean(ms)),
                     "timed_steps": n,
                     "setup_s": setup_s, "e2e": {"value": cells * nh / e2e_s, "unit": METRIC,
                                                 "note": "advance! of %d steps from rest, CD/CL returned" % nh},
                     "launches_per_step": G.launches_per_step(p), "nf": p.nf,
                     "cd_final": cd[-1].tolist(), "cl_final": cl[-1].tolist()}
        p.close()
    (cd32, cl32), (cd64, cl64) = hist["fp32_refined"], hist["fp64"]
    out["refined_vs_fp64"] = out["fp32_refined"]["value"] / out["fp64"]["value"]
    def errs(m0, m1):
        dcd, dcl = np.abs(cd32[m0:m1] - cd64[m0:m1]) / np.abs(cd64[m0:m1]), np.abs(cl32[m0:m1] - cl64[m0:m1])
        return {"cd_max_rel_err": float(np.max(dcd)),
                "cd_err_argmax_step": m0 + int(np.unravel_index(np.argmax(dcd), dcd.shape)[0]),
                "cl_err_rel_to_max_cl": float(np.max(dcl) / np.max(np.abs(cl64[m0:m1]))),
                "cl_err_rel_to_max_cd": float(np.max(dcl) / np.max(np.abs(cd64[m0:m1])))}
    out["accuracy"] = {"steps": nh, "forces": "CD and CL of each body", **errs(0, nh),
                       "by_range": {"%d-%d" % (m0, m1): errs(m0, m1)
                                    for m0, m1 in ((0, 10), (10, 100), (100, 1000), (1000, nh))},
                       "max_abs_cl": float(np.max(np.abs(cl64))), "max_abs_cd": float(np.max(np.abs(cd64)))}
    try:
        out["position_gradient"] = position_gradient_block(args, d, C5, "the same geometry: mean total lift "
                                                           "(last 100 of 400 steps), checkpoint every 100 steps, "
                                                           "8 seeded finite-difference directions (FP64)")
    except Exception as e:  # reported, not fatal
        out["position_gradient"] = {"error": str(e)[:300]}
    return out


def position_gradient_block(args, d, XB=XB, workload=XB_WORKLOAD):
    import ibpm_gpu as G
    g = G.make_grid(XB["h"], BOUNDARY, XB["mg"])
    ox, oy = XB["off"]

    def bodies(xb=None):
        bs = [G.make_cylinder(0.5, g.h, ox, 0.75 + oy, n=XB["nb"]), G.make_cylinder(0.5, g.h, ox, -0.75 + oy, n=XB["nb"])]
        if xb is not None:
            bs[0].xb, bs[1].xb = xb[:XB["nb"]].copy(), xb[XB["nb"]:].copy()
        return bs

    def problem(xb=None):
        return G.IBProblem(g, bodies(xb), XB["dt"], XB["Re"], device=d.local, sync_fields=False)
    rng = np.random.default_rng(XB["seed"])
    w0 = 1e-3 * rng.standard_normal((g.nx - 1, g.ny - 1))   # breaks the up-down symmetry: a nonzero lift

    def start(p):
        st = G.IBState(p)
        for a in (st.Gamma, st.q, st.psi, st.nonlin[0], st.nonlin[1], st.Fb):
            a[...] = 0.0
        st.Gamma[:, 0] = g.h ** 2 * w0.flatten(order="F")
        G.push_state(st, p)
        G.vort2flux(st, p)
        return st
    n, win = XB.get("adj_steps", XB["steps"]), XB["window"]

    def J_of(xb):
        p = problem(xb)
        st = start(p)
        _, cl = G.advance(st, p, 0.0, nsteps=n)
        p.close()
        return float(np.mean(np.sum(cl[-win:], axis=1)))
    prob = problem()
    xb0 = np.concatenate([b.xb for b in bodies()])
    st = start(prob)
    G.advance(st, prob, 0.0, nsteps=3)          # graph capture
    start(prob)
    G.adjoint_run(prob, n, XB["k"], win, w_cd=0.0, w_cl=1.0, want_xb=True)   # tape allocation, graph capture
    start(prob)
    prob.sync()
    t0 = time.perf_counter()
    G.advance(st, prob, 0.0, nsteps=n)
    t_fwd = time.perf_counter() - t0
    start(prob)
    prob.sync()
    t0 = time.perf_counter()
    res = G.adjoint_run(prob, n, XB["k"], win, w_cd=0.0, w_cl=1.0, want_xb=True)
    t_adj = time.perf_counter() - t0
    prob.close()
    eps = 1e-5 * g.h
    gn = float(np.linalg.norm(res.grad_xb))
    checks = []
    for _ in range(XB["ndir"]):
        dv = rng.standard_normal(xb0.shape)
        fd = (J_of(xb0 + eps * dv) - J_of(xb0 - eps * dv)) / (2 * eps)
        ad = float(np.sum(res.grad_xb * dv))
        checks.append({"fd": fd, "adjoint": ad, "err_over_norm": abs(fd - ad) / (gn * float(np.linalg.norm(dv))),
                       "rel_err": abs(fd - ad) / abs(fd)})
    return {"workload": workload, "precision": "fp64", "J": res.J, "grad_xb_norm": gn,
            "forward_s": t_fwd, "adjoint_run_s": t_adj, "adjoint_over_forward": t_adj / t_fwd,
            "reverse_over_forward": (t_adj - t_fwd) / t_fwd,
            "fd_eps": eps, "fd_checks": checks,
            "max_err_over_norm": max(c["err_over_norm"] for c in checks),
            "median_rel_err": float(np.median([c["rel_err"] for c in checks]))}


def adjoint_block(args, d):
    a64 = measure_adjoint(args, d, "fp64")
    a32 = measure_adjoint(args, d, "fp32_refined")
    gw64, gw32 = a64["grad_omega0"], a32["grad_omega0"]
    try:
        xb = position_gradient_block(args, d)
    except Exception as e:  # reported, not fatal
        xb = {"workload": XB_WORKLOAD, "error": str(e)[:300]}
    return {
        "workload": ADJ_WORKLOAD,
        "metric": "adjoint/forward cost",
        "value": (a64["adjoint_run_s"] - a64["forward_s"]) / a64["forward_s"],
        "reverse_over_forward": (a64["adjoint_run_s"] - a64["forward_s"]) / a64["forward_s"],
        "adjoint_over_forward": a64["adjoint_run_s"] / a64["forward_s"],
        "note": "value = reverse_over_forward = (wall(ibpm_adjoint_run) - wall(forward run)) / wall(forward "
                "run): the reverse sweep (recomputation from checkpoints + adjoint steps) per forward run; "
                "adjoint_over_forward also counts the forward pass with checkpoints that any gradient needs",
        "forward_s": a64["forward_s"], "adjoint_run_s": a64["adjoint_run_s"],
        "adjoint_step_ms": a64["adj_step_ms"], "forward_step_ms": a64["fwd_step_ms"],
        "adjoint_step_over_forward_step": a64["adj_step_ms"] / a64["fwd_step_ms"],
        "J": a64["J"], "J_forward_run": a64["J_forward"],
        "fd_check": {"eps": 1e-6, "fd": a64["fd"], "adjoint": a64["ad"],
                     "rel_err": abs(a64["fd"] - a64["ad"]) / abs(a64["fd"])},
        "grad_alpha": a64["grad_alpha"],
        "fp32_refined": {"adjoint_over_forward": a32["adjoint_run_s"] / a32["forward_s"],
                         "reverse_over_forward": (a32["adjoint_run_s"] - a32["forward_s"]) / a32["forward_s"],
                         "J_rel_diff_vs_fp64": abs(a32["J"] - a64["J"]) / abs(a64["J"]),
                         "grad_omega0_rel_diff_vs_fp64": float(np.max(np.abs(gw32 - gw64)) / np.max(np.abs(gw64))),
                         "note": "checked against the FP64 gradient: a central difference with eps = 1e-6 "
                                 "changes J by less than the refined forward run's own error"},
        "position_gradient": xb,
    }


# The batch workload: 64 independent static-body simulations, 16 each of
# nx = ny in {128, 192, 256, 384} (h = 4/nx, domain [-1, 3] x [-2, 2]), 3 to 5
# levels, Re uniform in [40, 200], cylinders (D = 1, ≈ 1 point per h) or NACA
# 4-digit sections (chord 1, thickness uniform in [0.08, 0.18], angle of
# attack uniform in [0, 15] deg about the leading edge, max panel ≈ h), dt =
# 0.2 h, FP32-refined; all drawn from one seed.
BATCH = dict(n=64, sizes=(128, 192, 256, 384), seed=5, steps=2000, one_lane_steps=200)
BATCH_WORKLOAD = ("64 independent simulations: nx=ny in {128,192,256,384} x16, h=4/nx, 3-5 levels, Re U[40,200], "
                  "cylinders or NACA 4-digit (t U[0.08,0.18], aoa U[0,15] deg), dt=0.2h, fp32_refined")


def naca_body(G, t, aoa, h):
    """A NACA 00xx section (chord 1, rotated by aoa about its leading edge)
    with boundary points ≈ h apart along the outline: the cosine-spaced
    outline of make_naca crowds points far closer than h at the leading edge
    and brings the two surfaces within h of each other near the trailing
    edge, which makes the Schur complement nearly singular.  The outline is
    sampled at uniform arc length h, dropping points closer than 0.75 h to
    one already kept (CD/CL do not depend on ds: it cancels in
    update_stress!)."""
    dense = G.make_naca(0.0, 4001, t, chord=1.0, aoa=aoa, pivot=(0.0, 0.0)).xb
    seg = np.sqrt(np.sum(np.diff(dense, axis=0) ** 2, axis=1))
    s = np.concatenate([[0.0], np.cumsum(seg)])
    n = max(8, int(round(s[-1] / h)))
    targets = np.linspace(0.0, s[-1], n, endpoint=False)
    pts = np.stack([np.interp(targets, s, dense[:, 0]), np.interp(targets, s, dense[:, 1])], axis=1)
    keep = []
    for p in pts:
        if all(np.hypot(*(p - q)) >= 0.75 * h for q in keep):
            keep.append(p)
    xb = np.array(keep)
    return G.RigidBody(xb=xb, ds=np.full(len(xb), s[-1] / len(xb)))


def batch_specs(G, seed=BATCH["seed"]):
    import math
    rng = np.random.default_rng(seed)
    specs = []
    for nx in [s for s in BATCH["sizes"] for _ in range(BATCH["n"] // len(BATCH["sizes"]))]:
        h = 4.0 / nx
        mg = int(rng.integers(3, 6))
        Re = float(rng.uniform(40.0, 200.0))
        g = G.make_grid(h, (-1.0, 3.0, -2.0, 2.0), mg)
        if rng.random() < 0.5:
            body = G.make_cylinder(0.5, g.h, 0.0, 0.0, n=int(math.floor(math.pi / g.h)))
        else:
            t = float(rng.uniform(0.08, 0.18))
            aoa = math.radians(float(rng.uniform(0.0, 15.0)))
            body = naca_body(G, t, aoa, g.h)
        specs.append(dict(grid=g, bodies=[body], dt=0.2 * g.h, Re=Re, precision="fp32_refined"))
    return specs


def batch_block(args, d):
    """Batch throughput: Σ_members nx·ny·mg per step over the device time of
    the workload's 2000 batch steps (graph launches, L2 flushed between
    steps), with the tuned lane count, transform plan and level chain, and
    over 200 steps with one lane (the members one after another, the same
    plan and chain); end to end, the 2000 steps through ibpm_batch_advance."""
    import ibpm_gpu as G
    specs = batch_specs(G)
    t0 = time.perf_counter()
    b = G.Batch(specs, lanes=0, device=d.local)
    setup_s = time.perf_counter() - t0
    cells = sum(sp["grid"].nx * sp["grid"].ny * sp["grid"].mg for sp in specs)
    K = BATCH["steps"]
    b.advance(40)                 # past the refined members' 32 two-sweep start-up steps
    tuned = b.lanes
    plan = b.plan
    chain = b.chain
    grouped = b.grouped
    ms = b.bench_steps(K, flush_l2=True)
    t_tuned = float(np.sum(ms)) / 1e3
    b.set_lanes(1)
    b.advance(2)
    K1 = BATCH["one_lane_steps"]
    ms1 = b.bench_steps(K1, flush_l2=True)
    t_seq = float(np.sum(ms1)) / 1e3 * K / K1
    b.set_lanes(tuned)            # end to end with the tuned lanes
    b.advance(2)
    t0 = time.perf_counter()
    forces = b.advance(K)
    e2e_s = time.perf_counter() - t0
    finite = all(np.all(np.isfinite(f[0])) for f in forces)
    b.close()
    return {"workload": BATCH_WORKLOAD, "metric": METRIC, "value": cells * K / t_tuned, "unit": METRIC,
            "steps": K, "lanes": tuned, "ms_per_batch_step": 1e3 * t_tuned / K,
            "transform_plan": {0: "latency (radix 4)", 1: "throughput (radix 8)"}.get(plan, plan),
            "level_chain": {0: "sequential", 1: "boundary transfer"}.get(chain, chain),
            "shared_launches": grouped,
            "one_lane": {"value": cells * K / t_seq, "ms_per_batch_step": 1e3 * t_seq / K, "steps": K1},
            "speedup_over_one_lane": t_seq / t_tuned,
            "e2e": {"value": cells * K / e2e_s, "unit": METRIC, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 16.0 * len(specs),
                    "note": "ibpm_batch_advance of K steps, CD/CL of every member returned to the host"},
            "setup_s": setup_s, "cells_per_step": cells, "forces_finite": finite}


# The reference's moving-grid benchmark (benchmarks/eldredge): a flat plate
# (L = 1, 51 points) on 400x200 cells x 5 levels, h = 0.02, Re = 100; the
# steady boundary layer (dt = 0.01, 10 001 steps) and from it the
# pitch-up/hold/down manoeuvre (dt = 1e-3, 10 001 steps, a = 11,
# t1..t4 = 1, 3, 4, 6, 45 degrees).  The reference reports 1098 s for the
# manoeuvre (benchmarks/eldredge/README.md:40-44, its own hardware).
ELDREDGE_WORKLOAD = ("Eldredge pitch manoeuvre, MovingGrid flat plate (51 pts) Re=100, 400x200 cells x 5 levels, "
                     "h=0.02, dt=1e-3, 10001 steps from the steady boundary layer (dt=1e-2, 10001 steps)")
ELDREDGE_REF_S = 1098.0
ELDREDGE_LAB_REF_S = 65867.0   # the same manoeuvre with the plate itself moving (lab frame)
GOLDEN_ELDREDGE = os.path.join(ROOT, "tests", "golden", "eldredge_pitch.json")
GOLDEN_ELDREDGE_MOTION = os.path.join(ROOT, "tests", "golden", "eldredge_pitch_motion.json")


def eldredge_motion():
    """θ(t), θ̇(t) of benchmarks/eldredge/pitch_maneuver.jl:11-20."""
    import math
    a, t1, t2, t3, t4 = 11.0, 1.0, 3.0, 4.0, 6.0
    amax = 45 * math.pi / 180

    def G(t):
        return np.log(np.cosh(a * (t - t1)) * np.cosh(a * (t - t4)) / (np.cosh(a * (t - t2)) * np.cosh(a * (t - t3))))

    gmax = float(np.max(G(np.arange(10001) * 1e-3)))
    ch, th = math.cosh, math.tanh

    def theta(t):   # scalar form of -amax G(t) / gmax (the host evaluates it every step)
        return -amax * math.log(ch(a * (t - t1)) * ch(a * (t - t4)) / (ch(a * (t - t2)) * ch(a * (t - t3)))) / gmax

    def theta_dot(t):
        return -amax * (a * (th(a * (t - t1)) - th(a * (t - t2)) - th(a * (t - t3)) + th(a * (t - t4)))) / gmax

    return theta, theta_dot


def eldredge_block(args, d):
    """The manoeuvre end to end through the public API (advance with the
    motion evaluated on the host every step, CD/CL returned), FP64, wall clock
    after the steady start state is computed; lab-frame CL/CD against the
    reference's own history (tests/golden/eldredge_pitch.json)."""
    import ibpm_gpu as G
    g = G.make_grid(0.02, (-1.5, 6.5, -2.0, 2.0), 5)
    steady = G.IBProblem(g, [G.make_plate(1.0, 0.0, g.h, 0.0, 0.0, n=51)], 1e-2, 100.0,
                         freestream=(1.0, 0.0, 0.0), device=d.local, sync_fields=False)
    st = G.IBState(steady)
    t0 = time.perf_counter()
    cd_s, _ = G.advance(st, steady, np.arange(10001) * 1e-2)
    steady_s = time.perf_counter() - t0
    G.pull_state(st, steady)
    steady.close()
    st0 = st.copy()               # the steady start, for the moving-body run below
    theta, theta_dot = eldredge_motion()
    mot = G.MovingGrid(U=lambda t: 1.0, V=lambda t: 0.0, theta=theta, theta_dot=theta_dot)
    pitch = G.IBProblem(g, [G.make_plate(1.0, 0.0, g.h, 0.0, 0.0, n=51, motion=mot)], 1e-3, 100.0,
                        freestream=(0.0, 0.0, 0.0), device=d.local, sync_fields=False)
    G.push_state(st, pitch)
    t = np.arange(10001) * 1e-3
    t0 = time.perf_counter()
    F1, F2 = G.advance(st, pitch, t)
    wall = time.perf_counter() - t0
    pitch.close()
    th = np.array([theta(tk) for tk in t])
    CD = F1[:, 0] * np.cos(th) - F2[:, 0] * np.sin(th)
    CL = F1[:, 0] * np.sin(th) + F2[:, 0] * np.cos(th)
    out = {"workload": ELDREDGE_WORKLOAD, "precision": "fp64", "steps": 10001, "seconds": wall,
           "steps_per_s": 10001 / wall, "level_cell_steps_per_s": 400 * 200 * 5 * 10001 / wall,
           "steady_start_seconds": steady_s, "steady_cd": float(cd_s[-1, 0]),
           "reference_published_seconds": ELDREDGE_REF_S,
           "reference_published_note": "Julia, body-fixed (MovingGrid) formulation, on the reference's own "
                                       "hardware (benchmarks/eldredge/README.md:40-44); not measured here",
           "timing": "wall clock around one advance call of 10001 steps: host evaluation of the motion, "
                     "one graph replay per step, per-step CD/CL returned"}
    try:
        with open(GOLDEN_ELDREDGE) as f:
            gold = json.load(f)
        k = gold["step_stride"]
        gcl, gcd = np.array(gold["CL_lab"]), np.array(gold["CD_lab"])
        out["vs_reference_history"] = {
            "cl_max_err_rel_to_peak": float(np.max(np.abs(CL[::k] - gcl)) / np.max(np.abs(gcl))),
            "cd_max_err_rel_to_peak": float(np.max(np.abs(CD[::k] - gcd)) / np.max(np.abs(gcd))),
            "source": gold["source"]}
    except OSError as e:
        out["vs_reference_history"] = {"error": str(e)[:200]}
    # the lab-frame form: the plate itself pitches (MotionFunction), E and B⁻¹
    # rebuilt every step (pitch_maneuver_motion.jl, 10 000 steps)
    try:
        mf = G.MotionFunction(xc=(lambda t: 0.0, lambda t: 0.0, theta), uc=(lambda t: 0.0, lambda t: 0.0, theta_dot))
        pb = G.IBProblem(g, [G.make_plate(1.0, 0.0, g.h, 0.0, 0.0, n=51, motion=mf)], 1e-3, 100.0,
                         freestream=(1.0, 0.0, 0.0), device=d.local, sync_fields=False)
        G.push_state(st0, pb)
        tm = np.arange(10000) * 1e-3
        t0 = time.perf_counter()
        CDm, CLm = G.advance(st0, pb, tm)
        wall_m = time.perf_counter() - t0
        pb.close()
        lab = {"seconds": wall_m, "steps": 10000, "steps_per_s": 10000 / wall_m,
               "reference_published_seconds": ELDREDGE_LAB_REF_S,
               "reference_published_note": "Julia, lab frame (MotionFunction: E and B⁻¹ per step, B by CG), on the "
                                           "reference's own hardware (benchmarks/eldredge/README.md:40-44)",
               "per_step": "kinematics, E weights, B rebuilt by 102 batched unit solves and inverted "
                           "(Gauss-Jordan), then the step"}
        with open(GOLDEN_ELDREDGE_MOTION) as f:
            gm = json.load(f)
        k = gm["step_stride"]
        gcl, gcd = np.array(gm["CL_lab"]), np.array(gm["CD_lab"])
        lab["vs_reference_history"] = {
            "cl_max_err_rel_to_peak": float(np.max(np.abs(CLm[::k, 0] - gcl)) / np.max(np.abs(gcl))),
            "cd_max_err_rel_to_peak": float(np.max(np.abs(CDm[::k, 0] - gcd)) / np.max(np.abs(gcd))),
            "source": gm["source"]}
        out["moving_body"] = lab
    except Exception as e:  # reported, not fatal
        out["moving_body"] = {"error": str(e)[:300]}
    return out


CONFIG_STEPS = 4000   # the workload's stated run length (t = 8)


def history(d, precision="fp64", scale=1.0, nsteps=CONFIG_STEPS):
    """CD/CL of nsteps steps (one advance call) from the vortex start with its
    amplitude scaled by ``scale``, and the final Γ.  With scale ≠ 1 on the
    FP64 path: the flow's own sensitivity to a change of the start state, the
    yardstick for the FP32-refined path's differences after many steps (the
    Re = 100 wake amplifies any difference)."""
    import ibpm_gpu as G
    g = G.make_grid(H, BOUNDARY, MG)
    prob = G.IBProblem(g, [G.make_cylinder(0.5, g.h, 0.0, 0.0, n=NB)], DT, RE, freestream=(1.0, 0.0, 0.0),
                       device=d.local, sync_fields=False, precision=precision)
    st = G.IBState(prob)
    st.Gamma[...] = scale * vortex_gamma(g.nx, g.ny, g.mg, g.h, g.offx, g.offy)
    G.push_state(st, prob, fields=("Gamma",))
    G.vort2flux(st, prob)
    cd, cl = G.advance(st, prob, 0.0, nsteps=nsteps)
    G.pull_state(st, prob)
    gamma = np.array(st.Gamma)
    prob.close()
    return cd[:, 0], cl[:, 0], gamma


def accuracy_block(d):
    """The FP32-refined path against the FP64 path over the workload's full
    4000 steps from the vortex start: CD relative to itself, CL relative to
    its own largest magnitude and on the force scale (max |CD|), by step
    range, beside the FP64 path's own divergence from a perturbed start."""
    cd32, cl32, g32 = history(d, "fp32_refined")
    cd64, cl64, g64 = history(d, "fp64")
    pcd, pcl, _ = history(d, "fp64", 1.0 + 1e-9)
    K = CONFIG_STEPS

    def errs(a, b, c, dd, m0, m1):
        return {"cd_max_rel_err": float(np.max(np.abs(a[m0:m1] - b[m0:m1]) / np.abs(b[m0:m1]))),
                "cl_max_abs_err": float(np.max(np.abs(c[m0:m1] - dd[m0:m1]))),
                "cl_err_rel_to_max_cl": float(np.max(np.abs(c[m0:m1] - dd[m0:m1])) / np.max(np.abs(dd[m0:m1]))),
                "cl_err_rel_to_max_cd": float(np.max(np.abs(c[m0:m1] - dd[m0:m1])) / np.max(np.abs(b[m0:m1])))}
    acc = {"reference": "the FP64 GPU path on the same start state (it matches the FP64 oracle to 1e-10)",
           "steps": K}
    acc.update(errs(cd32, cd64, cl32, cl64, 0, K))
    acc.update({
        "cl_err_argmax_step": int(np.argmax(np.abs(cl32 - cl64))),
        "cd_err_argmax_step": int(np.argmax(np.abs(cd32 - cd64) / np.abs(cd64))),
        "max_abs_cl": float(np.max(np.abs(cl64))), "max_abs_cd": float(np.max(np.abs(cd64))),
        "vorticity_rel_l2": float(np.linalg.norm(g32 - g64) / np.linalg.norm(g64)),
        "vorticity_rel_l2_finest": float(np.linalg.norm(g32[:, 0] - g64[:, 0]) / np.linalg.norm(g64[:, 0])),
        "by_range": {"%d-%d" % (m0, m1): {"refined": errs(cd32, cd64, cl32, cl64, m0, m1),
                                          "fp64_perturbed": errs(pcd, cd64, pcl, cl64, m0, m1)}
                     for m0, m1 in ((0, 10), (10, 100), (100, 1000), (1000, K))},
        "note": "by_range: max differences over steps [m0, m1); fp64_perturbed = the FP64 path started from "
                "the vortex amplitude x (1 + 1e-9); the first 10 steps are the impulsive start, during which "
                "the lift is 1e-6..1e-4 against CD up to 1640",
    })
    return acc


# Shedding: the same workload continued until the wake sheds periodically,
# in chunks of 5000 steps (t = 10 each), at most 100 000 steps (t = 200).
SHED = dict(chunk=5000, max_steps=100000, cycles=6, amp_tol=5e-3)


def shedding_cycles(cl, dt, cycles):
    """Period and amplitude of the last ``cycles`` full CL cycles: upward
    crossings of the mean of the last third, located by linear interpolation;
    the amplitude of a cycle is half its peak-to-peak.  None while fewer
    cycles exist."""
    x = cl - np.mean(cl[2 * len(cl) // 3:])
    i = np.nonzero((x[:-1] < 0) & (x[1:] >= 0))[0]
    if i.size < cycles + 1:
        return None
    tc = (i + x[i] / (x[i] - x[i + 1])) * dt
    amps = np.array([0.5 * (np.max(cl[a:b + 1]) - np.min(cl[a:b + 1])) for a, b in zip(i[:-1], i[1:])])
    per = np.diff(tc[-cycles - 1:])
    return {"period": float(np.mean(per)), "period_spread": float(np.ptp(per) / np.mean(per)),
            "cl_amplitude": float(np.mean(amps[-cycles:])), "amplitudes": amps,
            "window": [float(tc[-cycles - 1]), float(tc[-1])], "crossings": i}


def strouhal_block(args, d):
    """Vortex shedding of the workload: the FP64 path is continued until the
    CL amplitude of the last three cycles agrees to 0.5% (the limit cycle),
    then the FP32-refined path runs the same steps from the same start.  St =
    f D / U (D = 1, U = 1) from the mean period of the last cycles of each;
    the mean CD is taken over the same cycles."""
    import ibpm_gpu as G
    g = G.make_grid(H, BOUNDARY, MG)

    def run(precision, nmax, stop):
        prob = G.IBProblem(g, [G.make_cylinder(0.5, g.h, 0.0, 0.0, n=NB)], DT, RE, freestream=(1.0, 0.0, 0.0),
                           device=d.local, sync_fields=False, precision=precision, refine_sweeps=1)
        st = G.IBState(prob)
        st.Gamma[...] = vortex_gamma(g.nx, g.ny, g.mg, g.h, g.offx, g.offy)
        G.push_state(st, prob, fields=("Gamma",))
        G.vort2flux(st, prob)
        cds, cls = [], []
        n = 0
        t0 = time.perf_counter()
        while n < nmax:
            m = min(SHED["chunk"], nmax - n)
            cd, cl = G.advance(st, prob, n * DT, nsteps=m)
            cds.append(cd[:, 0])
            cls.append(cl[:, 0])
            n += m
            if stop and stop(np.concatenate(cls)):
                break
        wall = time.perf_counter() - t0
        prob.close()
        return np.concatenate(cds), np.concatenate(cls), wall

    def settled(cl):
        c = shedding_cycles(cl, DT, SHED["cycles"])
        if c is None or c["cl_amplitude"] < 1e-2:
            return False
        a = c["amplitudes"][-3:]
        return bool(np.ptp(a) / np.mean(a) < SHED["amp_tol"])

    cd64, cl64, wall64 = run("fp64", SHED["max_steps"], settled)
    n = cd64.size
    cd32, cl32, wall32 = run("fp32_refined", n, None)
    out = {"workload": WORKLOAD + ", continued to the periodic wake", "steps": n, "t_end": n * DT,
           "limit_cycle": settled(cl64), "seconds": {"fp64": wall64, "fp32_refined": wall32},
           "reference": "the FP64 GPU path (it matches the FP64 oracle to 1e-10 per step)"}
    res = {}
    for name, cd, cl in (("fp64", cd64, cl64), ("fp32_refined", cd32, cl32)):
        c = shedding_cycles(cl, DT, SHED["cycles"])
        if c is None:
            res[name] = None
            continue
        a, b = c["crossings"][-SHED["cycles"] - 1], c["crossings"][-1]
        res[name] = {"strouhal": 1.0 / c["period"], "period_spread": c["period_spread"],
                     "cl_amplitude": c["cl_amplitude"], "cd_mean": float(np.mean(cd[a:b])),
                     "window_t": c["window"]}
    out.update(res)
    if res.get("fp64") and res.get("fp32_refined"):
        r, f = res["fp32_refined"], res["fp64"]
        out["strouhal_rel_err"] = abs(r["strouhal"] - f["strouhal"]) / f["strouhal"]
        out["cl_amplitude_rel_err"] = abs(r["cl_amplitude"] - f["cl_amplitude"]) / f["cl_amplitude"]
        out["cd_mean_rel_err"] = abs(r["cd_mean"] - f["cd_mean"]) / f["cd_mean"]
    out["note"] = ("St from the mean period of the last %d CL cycles (upward crossings of the mean, linear "
                   "interpolation); the phase of the two runs drifts apart, the limit cycle does not"
                   % SHED["cycles"])
    return out


def run_ours(args, d):
    K = args.steps
    sampler = ClockSampler(d.local)
    r32 = measure(args, d, "fp32_refined", sampler)
    r64 = measure(args, d, "fp64")
    g, cells = r32["g"], r32["cells"]
    value = d.world * cells * K / (r32["total_ms"] / 1e3)
    value64 = d.world * cells * K / (r64["total_ms"] / 1e3)

    def e2e_of(r):
        return {"value": d.world * cells * K / r["e2e_s"], "unit": METRIC,
                "h2d_bytes_per_step": r["state_bytes"] / K,
                "d2h_bytes_per_step": (r["state_bytes"] + 16 * r["bodies"] * K) / K,
                "note": "state uploaded once and downloaded once (amortised over the K steps); each "
                        "advance! call returns CD/CL to the host"}

    prof = r32["prof"]
    dom = max(prof, key=lambda k: prof[k][0])
    dms, dbytes, dcalls = prof[dom]
    peak, peak_kind = read_peaks()
    achieved = dbytes / (dms / 1e3) / 1e9
    step_s = (r32["total_ms"] / 1e3) / K
    step_s64 = (r64["total_ms"] / 1e3) / K
    launch_bytes = sum(v[1] for v in prof.values()) / 4.0
    launch_bytes64 = sum(v[1] for v in r64["prof"].values()) / 4.0
    bstep64 = step_bytes_model(g.nx, g.ny, g.mg, r64["nf"])
    accuracy = None
    if not args.no_accuracy:
        try:
            accuracy = accuracy_block(d)
        except Exception as e:  # reported, not fatal
            accuracy = {"error": str(e)[:300]}
    out = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": d.world, "steps": K,
        "warmup": args.warmup, "ms_per_step": r32["total_ms"] / K, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 transforms / f64 state, residuals, forces",
        "data": "synthetic",
        "config": {"workload": WORKLOAD, "precision": "fp32_refined (1 FP64-residual sweep per refined solve: "
                   "the projection and the final vort2flux!, warm start; FP64 trial solve and trial "
                   "vort2flux!)",
                   "l2": "flushed between steps (512 MiB write outside the timed event pairs)", "parallelism": "replicas x%d" % d.world,
                   "graph": "one CUDA graph replay per step",
                   "warmup_replays": "max(W, 40): the FP32-refined path's 32 two-sweep start-up steps are not timed",
                   "transform_plans": "radix-4 latency plan on single-level launches; multi-level launches "
                                      "automatic: radix 8 from 4 slabs on (the all-level launches)"},
        "e2e": e2e_of(r32),
        "gpu_launches": r32["lps"] * K,
        "fp64_plain": {"value": value64, "ms_per_step": r64["total_ms"] / K, "e2e": e2e_of(r64),
                       "gpu_launches": r64["lps"] * K,
                       "step_roofline": {"model_bytes_per_step": bstep64, "achieved_GBs": bstep64 / step_s64 / 1e9,
                                         "frac": bstep64 / step_s64 / 1e9 / peak,
                                         "launch_bytes_per_step": launch_bytes64},
                       "kernels": {k: {"ms_per_step": v[0] / 4.0, "launches_per_step": v[2] / 4.0}
                                   for k, v in r64["prof"].items()}},
        "refined_vs_fp64": value / value64,
        "accuracy": accuracy,
        "roofline": {"kernel": dom, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)"
                     if peak_kind == "measured" else "fallback 6.65 TB/s",
                     "traffic": read_traffic(dom), "launches_per_step": dcalls / 4.0,
                     "bytes_per_launch": dbytes / dcalls, "avg_launch_us": 1e3 * dms / dcalls},
        "step_roofline": {"launch_bytes_per_step": launch_bytes, "achieved_GBs": launch_bytes / step_s / 1e9,
                          "frac": launch_bytes / step_s / 1e9 / peak},
        "kernels": {k: {"ms_per_step": v[0] / 4.0, "GBs": (v[1] / (v[0] / 1e3) / 1e9) if v[0] > 0 else 0,
                        "launches_per_step": v[2] / 4.0} for k, v in prof.items()},
        "clocks": r32["clocks"],
    }
    if not args.no_adjoint:
        out["adjoint"] = adjoint_block(args, d)
    if not args.no_large:
        try:
            out["two_cylinders_1024"] = config5_block(args, d)
        except Exception as e:  # reported, not fatal
            out["two_cylinders_1024"] = {"workload": C5_WORKLOAD, "error": str(e)[:300]}
    if not args.no_eldredge:
        try:
            out["eldredge"] = eldredge_block(args, d)
        except Exception as e:  # reported, not fatal
            out["eldredge"] = {"workload": ELDREDGE_WORKLOAD, "error": str(e)[:300]}
    if d.world == 1 and not args.no_strouhal:
        try:
            out["strouhal"] = strouhal_block(args, d)
        except Exception as e:  # reported, not fatal
            out["strouhal"] = {"error": str(e)[:300]}
    if not args.no_batch:
        try:
            out["batch"] = batch_block(args, d)
        except Exception as e:  # reported, not fatal: the headline line still prints
            out["batch"] = {"workload": BATCH_WORKLOAD, "error": str(e)[:300]}
    if d.world == 1 and not args.no_cpu:
        try:
            rate, secs = cpu_step_rate(args.cpu_steps, os.cpu_count() or 1)
            out["cpu_baseline"] = {"value": rate, "unit": METRIC, "cores": os.cpu_count() or 1, "kind": "port",
                                   "sample": "%d steps of the same workload in oracle/ibpm_ref.py (%.1f s), "
                                             "scipy.fft on all host threads; B^-1 replaced by a seeded dense "
                                             "matrix of the same size" % (args.cpu_steps, secs)}
            # the reference's own FFTW plans run on one thread
            n1 = max(1, args.cpu_steps // 4)
            rate1, secs1 = cpu_step_rate(n1, 1)
            out["cpu_baseline"]["single_thread"] = {"value": rate1, "cores": 1,
                                                    "sample": "%d steps, scipy.fft on one thread (%.1f s)"
                                                              % (n1, secs1)}
        except Exception as e:  # the CPU leg is a reported baseline only
            out["cpu_baseline"] = {"value": None, "error": str(e)[:200]}
    if d.rank == 0:
        print(json.dumps(out))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-steps", type=int, default=20)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--no-eldredge", action="store_true")
    ap.add_argument("--no-strouhal", action="store_true")
    ap.add_argument("--no-large", action="store_true")
    ap.add_argument("--no-accuracy", action="store_true")
    args = ap.parse_args()
    d = Dist()
    try:
        if args.impl == "reference":
            return run_reference(args, d)
        return run_ours(args, d)
    finally:
        d.close()


if __name__ == "__main__":
    sys.exit(main())
