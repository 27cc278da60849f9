"""ibpm_lap_inv_noalloc: the inverse-Laplacian solve for callers that cannot
allocate device memory (their memory belongs to a pool or arena they do not
share).  The test is such a caller's stand-in: it owns its device buffers
(allocated here through the CUDA runtime, not by the library), calls the
allocation-free entry point twice in a row (different sizes and inputs, so the
shared scratch is reused and the transform tables are rebuilt) and checks each
result against the existing entry point that computes the same operator —
ψ = Δ⁻¹Γ from ibpm_vort2flux on a one-level problem — within the parity
tolerance of the other GPU tests."""
import ctypes
import glob
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
TOL = 1e-10


def cudart():
    cands = sorted(glob.glob("/usr/local/cuda/lib64/libcudart.so*"))
    lib = ctypes.CDLL(cands[-1])
    lib.cudaMalloc.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.c_size_t]
    lib.cudaMemcpy.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int]
    lib.cudaFree.argtypes = [ctypes.c_void_p]
    return lib


def reference_psi(nx_bnd, G_in):
    """ψ = Δ⁻¹ Γ through the existing entry point (one-level problem)."""
    import ibpm_gpu as G
    h, bnd, body = nx_bnd
    g = G.make_grid(h, bnd, 1)
    prob = G.IBProblem(g, [body(G, g.h)], 0.01, 100.0)
    st = G.IBState(prob)
    st.Gamma[:, 0] = G_in.flatten(order="F")
    G.push_state(st, prob, fields=("Gamma",))
    G.vort2flux(st, prob)
    out = st.psi[:, 0].reshape((g.nx - 1, g.ny - 1), order="F").copy()
    prob.close()
    return g, out


CASES = [
    ((0.0625, (-2.0, 2.0, -2.0, 2.0), lambda G, h: G.make_cylinder(0.5, h, 0.0, 0.0, n=40)), 1),
    ((1.0 / 32, (-2.0, 2.0, -1.0, 1.0), lambda G, h: G.make_cylinder(0.25, h, 0.0, 0.0, n=24)), 2),
]


def test_noalloc_matches_existing_entry_point_twice():
    import ibpm_gpu as G
    lib = G.load_library()
    lib.ibpm_lap_inv_noalloc.restype = ctypes.c_int
    lib.ibpm_lap_inv_noalloc.argtypes = [ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p,
                                         ctypes.c_void_p]
    rt = cudart()
    H2D, D2H = 1, 2
    for call, (spec, seed) in enumerate(CASES):
        g = G.make_grid(spec[0], spec[1], 1)
        rng = np.random.default_rng(seed)
        Gin = np.asfortranarray(rng.standard_normal((g.nx - 1, g.ny - 1)))
        nbytes = Gin.nbytes
        d_in, d_out = ctypes.c_void_p(), ctypes.c_void_p()
        assert rt.cudaMalloc(ctypes.byref(d_in), nbytes) == 0
        assert rt.cudaMalloc(ctypes.byref(d_out), nbytes) == 0
        try:
            assert rt.cudaMemcpy(d_in, Gin.ctypes.data, nbytes, H2D) == 0
            rc = lib.ibpm_lap_inv_noalloc(g.nx, g.ny, d_in, d_out, None)
            assert rc == 0, lib.ibpm_last_error(None)
            out = np.empty_like(Gin, order="F")
            assert rt.cudaMemcpy(out.ctypes.data, d_out, nbytes, D2H) == 0   # waits for the solve
        finally:
            rt.cudaFree(d_in)
            rt.cudaFree(d_out)
        _, ref = reference_psi(spec, Gin)
        err = np.max(np.abs(out - ref)) / np.max(np.abs(ref))
        assert err < TOL, (call, err)


def test_noalloc_rejects_oversize():
    import ibpm_gpu as G
    lib = G.load_library()
    lib.ibpm_lap_inv_noalloc.restype = ctypes.c_int
    lib.ibpm_lap_inv_noalloc.argtypes = [ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p,
                                         ctypes.c_void_p]
    rc = lib.ibpm_lap_inv_noalloc(1024, 1024, ctypes.c_void_p(16), ctypes.c_void_p(16), None)
    assert rc == G.IBPM_ERR_INVALID
    assert b"at most 512" in lib.ibpm_last_error(None)
