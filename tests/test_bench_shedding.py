"""The shedding analysis of bench.py (host logic, CPU): the period, amplitude
and limit-cycle test it applies to a CL history, on synthetic signals whose
answers are known."""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _signal(st=0.1672, amp=0.33, dt=0.002, n=60000, growth=0.15, t_half=50.0, mean=1e-3):
    t = np.arange(n) * dt
    a = amp / (1.0 + np.exp(-growth * (t - t_half)))     # grows, then saturates
    return a * np.sin(2 * np.pi * st * t + 0.3) + mean


def test_period_and_amplitude_of_a_saturated_wake():
    import bench
    c = bench.shedding_cycles(_signal(t_half=30.0), 0.002, 6)     # saturated from t ≈ 90 on
    assert abs(1.0 / c["period"] - 0.1672) / 0.1672 < 1e-4
    assert abs(c["cl_amplitude"] - 0.33) / 0.33 < 1e-3
    assert c["period_spread"] < 1e-3
    assert c["window"][0] < c["window"][1]


def test_too_few_cycles_give_none():
    import bench
    assert bench.shedding_cycles(_signal(n=1000), 0.002, 6) is None


def test_growing_wake_is_not_a_limit_cycle():
    """The amplitude test of the bench's stopping rule: the last three cycles
    must agree to 0.5%, which a wake still growing about 8% a cycle does not
    (its period is still found)."""
    import bench
    c = bench.shedding_cycles(_signal(growth=0.015, t_half=200.0), 0.002, 6)
    assert abs(1.0 / c["period"] - 0.1672) / 0.1672 < 1e-3
    a = c["amplitudes"][-3:]
    assert np.ptp(a) / np.mean(a) > bench.SHED["amp_tol"]
    c = bench.shedding_cycles(_signal(t_half=30.0), 0.002, 6)
    a = c["amplitudes"][-3:]
    assert np.ptp(a) / np.mean(a) < bench.SHED["amp_tol"]
