"""The C ABI library: it loads without a GPU and exports every entry point
that include/ibpm_gpu.h declares; create fails cleanly without a device."""
import ctypes
import os
import re

import numpy as np
import pytest

import ibpm_gpu as G

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(ROOT, "include", "ibpm_gpu.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(ibpm_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_header_symbols():
    lib = ctypes.CDLL(G.LIB_PATH)
    names = header_functions()
    assert "ibpm_advance" in names and "ibpm_create" in names
    for n in names:
        assert hasattr(lib, n), n


def test_version_string():
    assert "sm_100a" in G.version()


def test_desc_layout_matches_header():
    # the ctypes mirror must have the C struct's field order
    src = open(os.path.join(ROOT, "include", "ibpm_gpu.h")).read()
    body = src[src.index("typedef struct ibpm_problem_desc"):src.index("} ibpm_problem_desc;")]
    body = re.sub(r"//.*|/\*.*?\*/", "", body, flags=re.S)
    fields = re.findall(r"([A-Za-z_][A-Za-z0-9_]*)\s*(?:\[\d+\])?\s*[,;]", body)
    assert [f for f, _ in G.ProblemDesc._fields_] == fields


def test_host_setup_matches_oracle():
    from oracle import ibpm_ref as R
    for h, bnd in [(0.02, (-1.0, 3.0, -2.0, 2.0)), (0.01, (-1.0, 4.12, -2.56, 2.56))]:
        a, b = G.make_grid(h, bnd, 3), R.make_grid(h, bnd, 3)
        assert (a.nx, a.ny, a.h, a.offx, a.offy) == (b.nx, b.ny, b.h, b.offx, b.offy)
    c1, c2 = G.make_cylinder(0.5, 0.02, 0.0, 0.75, n=157), R.make_cylinder(0.5, 0.02, 0.0, 0.75, n=157)
    assert np.array_equal(c1.xb, c2.xb) and np.array_equal(c1.ds, c2.ds)
    p1, p2 = G.make_plate(1.0, 0.0, 0.02, 0.0, 0.0, n=51), R.make_plate(1.0, 0.0, 0.02, 0.0, 0.0, n=51)
    assert np.array_equal(p1.xb, p2.xb)
    n1 = G.make_naca(0.0, 80, 0.12, aoa=0.1)
    n2 = R.make_naca(0.0, 80, 0.12, aoa=0.1)
    assert np.allclose(n1.xb, n2.xb, rtol=0, atol=0) and np.allclose(n1.ds, n2.ds, rtol=0, atol=0)


def test_create_without_gpu_fails_loudly():
    import subprocess
    import sys
    code = ("import sys; sys.path.insert(0, %r); import ibpm_gpu as G\n"
            "g = G.make_grid(0.0625, (-2., 2., -2., 2.), 2)\n"
            "try:\n    G.IBProblem(g, [G.make_cylinder(0.5, g.h, 0, 0, n=40)], 0.01, 40.)\n"
            "except G.IBPMError as e:\n    print('ERR', e.code); sys.exit(0)\n"
            "print('CREATED')\n") % os.path.join(ROOT, "ibpm.jl_b200", "python")
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, env=env, timeout=120)
    assert out.returncode == 0, out.stderr
    assert "ERR -2" in out.stdout


def test_create_validates_precision_before_touching_a_device():
    """An unknown precision mode or sweep count is rejected with
    IBPM_ERR_INVALID by argument checking alone (no GPU needed)."""
    import ibpm_gpu as G
    g = G.make_grid(0.0625, (-2., 2., -2., 2.), 2)
    body = G.make_cylinder(0.5, g.h, 0, 0, n=40)
    with pytest.raises(G.IBPMError) as e:
        G.IBProblem(g, [body], 0.01, 40., precision="fp32_refined", refine_sweeps=-1)
    assert e.value.code == G.IBPM_ERR_INVALID
    with pytest.raises(G.IBPMError) as e:
        G.IBProblem(g, [body], 0.01, 40., precision="fp16")
    assert e.value.code == G.IBPM_ERR_INVALID
