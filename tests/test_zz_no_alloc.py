"""ibpm_lap_inv_noalloc: the inverse-Laplacian solve for callers that cannot
allocate device memory.  Such a caller's device memory belongs to an allocator
it does not control (a Julia or Python runtime with its own caching pool, an
application with a fixed memory budget), so it hands the library its own
input and output buffers and expects no allocation behind its back.

The test is that caller: it owns its device buffers (allocated here through
the CUDA runtime, not by the library) and calls the entry point several times
in a row at different sizes, so the shared scratch is reused and the tables of
an earlier size are read again after another size ran.  Each result is checked
against the oracle's Δ⁻¹ (dst_inv with lap_eigs and the 1/(4 nx ny) scale of
get_lap_inv, src/fluid-operators/laplacian.jl:14-41) within the parity
tolerance of the other GPU tests.  A repeated call of one size must leave the
device's free memory unchanged."""
import ctypes
import glob
from types import SimpleNamespace

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
TOL = 1e-10
H2D, D2H = 1, 2


def cudart():
    cands = sorted(glob.glob("/usr/local/cuda/lib64/libcudart.so*"))
    lib = ctypes.CDLL(cands[-1])
    lib.cudaMalloc.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.c_size_t]
    lib.cudaMemcpy.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int]
    lib.cudaFree.argtypes = [ctypes.c_void_p]
    lib.cudaMemGetInfo.argtypes = [ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_size_t)]
    lib.cudaStreamCreate.argtypes = [ctypes.POINTER(ctypes.c_void_p)]
    lib.cudaStreamSynchronize.argtypes = [ctypes.c_void_p]
    lib.cudaStreamDestroy.argtypes = [ctypes.c_void_p]
    lib.cudaDeviceSynchronize.argtypes = []
    return lib


def entry_point():
    import ibpm_gpu as G
    lib = G.load_library()
    lib.ibpm_lap_inv_noalloc.restype = ctypes.c_int
    lib.ibpm_lap_inv_noalloc.argtypes = [ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p,
                                         ctypes.c_void_p]
    return lib


def oracle_lap_inv(b):
    from oracle import ibpm_ref as R
    g = SimpleNamespace(nx=b.shape[0] + 1, ny=b.shape[1] + 1)
    return R.dst_inv(b, R.lap_eigs(g), R.lap_inv_scale(g))


class DeviceField:
    """One caller-owned device buffer of an (nx-1)×(ny-1) column-major field."""

    def __init__(self, rt, nbytes):
        self.rt, self.nbytes, self.ptr = rt, nbytes, ctypes.c_void_p()
        assert rt.cudaMalloc(ctypes.byref(self.ptr), nbytes) == 0

    def free(self):
        self.rt.cudaFree(self.ptr)


def free_bytes(rt):
    free, total = ctypes.c_size_t(), ctypes.c_size_t()
    assert rt.cudaMemGetInfo(ctypes.byref(free), ctypes.byref(total)) == 0
    return free.value


def solve(lib, rt, nx, ny, seed, stream=None):
    rng = np.random.default_rng(seed)
    b = np.asfortranarray(rng.standard_normal((nx - 1, ny - 1)))
    d_in, d_out = DeviceField(rt, b.nbytes), DeviceField(rt, b.nbytes)
    try:
        assert rt.cudaMemcpy(d_in.ptr, b.ctypes.data, b.nbytes, H2D) == 0
        rc = lib.ibpm_lap_inv_noalloc(nx, ny, d_in.ptr, d_out.ptr, stream)
        assert rc == 0, lib.ibpm_last_error(None)
        if stream is not None:
            assert rt.cudaStreamSynchronize(stream) == 0
        out = np.empty_like(b, order="F")
        assert rt.cudaMemcpy(out.ctypes.data, d_out.ptr, b.nbytes, D2H) == 0
    finally:
        d_in.free()
        d_out.free()
    return b, out


def check(b, out, what):
    ref = oracle_lap_inv(b)
    err = np.max(np.abs(out - ref)) / np.max(np.abs(ref))
    assert err < TOL, (what, err)


def test_noalloc_matches_oracle_on_calls_in_a_row():
    lib, rt = entry_point(), cudart()
    # 64², then 128×64 (another x length), then the 512² limit
    for call, (nx, ny) in enumerate([(64, 64), (128, 64), (512, 512)]):
        b, out = solve(lib, rt, nx, ny, seed=call + 1)
        check(b, out, (call, nx, ny))
    # on a stream of the caller's own: a new y length, then back to the first
    # x length, whose tables were set up before the other sizes ran
    stream = ctypes.c_void_p()
    assert rt.cudaStreamCreate(ctypes.byref(stream)) == 0
    try:
        for call, (nx, ny) in enumerate([(64, 128), (64, 64)]):
            b, out = solve(lib, rt, nx, ny, seed=10 + call, stream=stream)
            check(b, out, ("stream", call, nx, ny))
    finally:
        rt.cudaStreamDestroy(stream)


def test_noalloc_allocates_nothing():
    lib, rt = entry_point(), cudart()
    nx = ny = 256
    rng = np.random.default_rng(5)
    b = np.asfortranarray(rng.standard_normal((nx - 1, ny - 1)))
    d_in, d_out = DeviceField(rt, b.nbytes), DeviceField(rt, b.nbytes)
    try:
        assert rt.cudaMemcpy(d_in.ptr, b.ctypes.data, b.nbytes, H2D) == 0
        assert lib.ibpm_lap_inv_noalloc(nx, ny, d_in.ptr, d_out.ptr, None) == 0
        assert rt.cudaDeviceSynchronize() == 0
        before = free_bytes(rt)
        for _ in range(2):
            assert lib.ibpm_lap_inv_noalloc(nx, ny, d_in.ptr, d_out.ptr, None) == 0
        assert rt.cudaDeviceSynchronize() == 0
        after = free_bytes(rt)
        out = np.empty_like(b, order="F")
        assert rt.cudaMemcpy(out.ctypes.data, d_out.ptr, b.nbytes, D2H) == 0
    finally:
        d_in.free()
        d_out.free()
    assert after == before, (before, after)
    check(b, out, "repeated")


def test_noalloc_rejects_oversize():
    import ibpm_gpu as G
    lib = entry_point()
    rc = lib.ibpm_lap_inv_noalloc(1024, 1024, ctypes.c_void_p(16), ctypes.c_void_p(16), None)
    assert rc == G.IBPM_ERR_INVALID
    assert b"at most 512" in lib.ibpm_last_error(None)
