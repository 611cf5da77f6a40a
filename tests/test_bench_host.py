"""Host logic of the benchmark that needs no GPU: the calibration that sets
the geometric theta and the learned budget to the loosest value within the
force-error target (a fake engine stands in for the device)."""
from __future__ import annotations

import numpy as np
import pytest


class FakeEngine:
    """rms error = (value / scale)^power * 1e-3 for the parameter being set."""

    def __init__(self, scale, power):
        self.scale, self.power, self.v = scale, power, None
        self.evaluations = 0

    def set_param(self, param, value):
        self.v = value

    def set_state(self, b, old_acc=False):
        pass

    def step(self, n, dt, eps, flags):
        pass

    def force_error(self, samples, seed, eps):
        self.evaluations += 1
        rms = (self.v / self.scale) ** self.power * 1e-3
        return (0.8 * rms, 5 * rms, rms)


def test_calibrate_refines_between_grid_points():
    import bench

    eng = FakeEngine(0.7, 4.0)
    best, rms, scanned = bench.calibrate(eng, None, None, 1, bench.THETA_GRID, 0, 0,
                                         lambda m: None)
    # coarse grid: 0.6875 passes, 0.7 does not; refined: 0.69, 0.6925, 0.695 pass, 0.6975 not
    assert best == pytest.approx(0.695)
    assert rms <= bench.CALIBRATION_TARGET
    assert eng.v == pytest.approx(0.695)
    values = [v for v, _ in scanned]
    assert values[-1] == pytest.approx(0.6975)
    assert all(r <= bench.CALIBRATION_TARGET for v, r in scanned if v <= 0.695 + 1e-12)


def test_calibrate_budget_grid_and_no_passing_value():
    import bench

    # learned budget: error grows with the budget (log10); the loosest value
    # within the target lies between -3.3 and -3.25
    eng = FakeEngine(1.0, 1.0)
    eng.force_error = lambda s, seed, e: (0, 0, 1e-3 * 10 ** (3.27 + eng.v))
    best, rms, _ = bench.calibrate(eng, None, None, 8, bench.BUDGET_GRID, 0, 0, lambda m: None)
    assert -3.3 <= best < -3.25 and rms <= bench.CALIBRATION_TARGET
    assert 1e-3 * 10 ** (3.27 + best + 0.01) > bench.CALIBRATION_TARGET
    # nothing within the target: the first grid value is left set, no value returned
    eng2 = FakeEngine(0.1, 1.0)
    best2, rms2, scanned2 = bench.calibrate(eng2, None, None, 1, bench.THETA_GRID, 0, 0,
                                            lambda m: None)
    assert best2 is None and rms2 is None
    assert eng2.v == bench.THETA_GRID[0] and len(scanned2) == len(bench.THETA_GRID)


def test_audit_bound_sits_above_the_target():
    import bench

    assert bench.CALIBRATION_TARGET < bench.RMS_TARGET < bench.AUDIT_RMS_BOUND
    assert bench.AUDIT_SAMPLES == 1024
    assert np.isclose(bench.AUDIT_RMS_BOUND, 1.2e-3)
