"""The Python example that the integration guide quotes (tests/integration_example.py),
run as written: the documented calls stay the library's calls."""
import runpy
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


def test_python_example_runs():
    ns = runpy.run_path(os.path.join(HERE, "integration_example.py"))
    G = ns["G"]
    assert ns["cd"].shape == (1000, 1) and np.all(np.isfinite(ns["cd"]))
    assert np.isfinite(ns["res"].J) and ns["res"].grad_xb.shape == (314, 2)
    assert ns["F1"].shape == (1000, 1) and np.all(np.isfinite(ns["F2"]))
    assert ns["CD"].shape == (100, 1) and np.all(np.isfinite(ns["CL"]))
    th = ns["theta"](99e-3)
    x0 = np.linspace(0.0, 1.0, 51)
    assert np.allclose(ns["xb"][:, 0], np.cos(th) * x0, atol=1e-14)
    assert np.allclose(ns["xb"][:, 1], np.sin(th) * x0, atol=1e-14)
    assert len(ns["histories"]) == 3 and all(np.all(np.isfinite(h[0])) for h in ns["histories"])
    for name in ("prob", "prob32", "pp", "pb"):
        ns[name].close()
    ns["batch"].close()
    assert G.version().startswith("ibpm_gpu")
