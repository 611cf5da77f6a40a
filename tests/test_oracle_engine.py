"""The oracle's FP64 direct sums, Verlet / Yoshida4 steps and energies
against the reference's own simulation Engine and EnergyTracker, compiled in
place into oracle/_ref (engine/src/sim/engine.cpp, engine/src/profile/
energy_tracker.cpp), and the three direct-sum orders of the desktop app's
CPU backends against each other.  CPU only.

Findings pinned here:
  * the native engine's CPU brute force (Engine::compute_cpu_brute_forces,
    engine.cpp:649-674) multiplies m * ((inv*inv)*inv), as the SIMD and
    single-thread C# backends do, not CpuParallelBackend's ((m*inv)*inv)*inv;
    its forces and trajectories are bit-identical to the SIMD-order
    restatement, not to the CpuParallel one;
  * the three orders agree to a few ulp (relative 1e-14), well inside the
    reference's own SIMD parity bound of 1e-12
    (tests/CelestialMechanics.Physics.Tests/SIMDParityTests.cs:62-100).
"""
from __future__ import annotations

import numpy as np
import pytest

from helpers import rel_err
from nbody_b200 import scenarios


def _state(n, seed, inactive_every=0):
    b = scenarios.plummer(n, 1.0, 1.0, seed=seed)
    if inactive_every:
        b.active[3::inactive_every] = 0
    d = {k: getattr(b, k) for k in ("px", "py", "pz", "vx", "vy", "vz", "ax", "ay", "az",
                                     "mass", "active")}
    d["radius"] = None
    return d


@pytest.mark.parametrize("n,inactive", [(1000, 0), (517, 7)])
def test_engine_brute_force_equals_simd_order(ref_lib, n, inactive):
    """One CPU_BruteForce Engine::step with dt = 0 leaves positions and
    velocities as they were and leaves the forces in acc."""
    d = _state(n, 21, inactive)
    got = ref_lib.ref_engine_steps(d, 1e-4, 0.0, 1)
    want = ref_lib.direct_forces_order(d["px"], d["py"], d["pz"], d["mass"], d["active"], 1e-4,
                                       ref_lib.ORDER_SIMD)
    for k, w in zip(("ax", "ay", "az"), want):
        np.testing.assert_array_equal(got[k], w, err_msg=k)
    par = ref_lib.direct_forces(d["px"], d["py"], d["pz"], d["mass"], d["active"], 1e-4)
    # CpuParallelBackend rounds the coefficient differently: not the same bits
    assert any(not np.array_equal(got[k], p) for k, p in zip(("ax", "ay", "az"), par))


def test_engine_leapfrog_trajectory_equals_oracle(ref_lib):
    """50 CPU_BruteForce Leapfrog_KDK steps of the reference Engine and of
    the oracle's Verlet restatement in the SIMD / engine order: bit-identical."""
    d = _state(300, 22, 11)
    a0 = ref_lib.direct_forces_order(d["px"], d["py"], d["pz"], d["mass"], d["active"], 1e-4,
                                     ref_lib.ORDER_SIMD)
    d["ax"], d["ay"], d["az"] = a0
    got = ref_lib.ref_engine_steps(d, 1e-4, 1e-3, 50)
    want = ref_lib.verlet_direct(d, 1e-4, 1e-3, 50, order=ref_lib.ORDER_SIMD)
    for k in ("px", "py", "pz", "vx", "vy", "vz", "ax", "ay", "az"):
        np.testing.assert_array_equal(got[k], want[k], err_msg=k)


def test_engine_yoshida4_trajectory_equals_oracle(ref_lib):
    d = _state(200, 23)
    d["ax"], d["ay"], d["az"] = ref_lib.direct_forces_order(
        d["px"], d["py"], d["pz"], d["mass"], d["active"], 1e-4, ref_lib.ORDER_SIMD)
    got = ref_lib.ref_engine_steps(d, 1e-4, 1e-3, 20, integrator=1)
    want = ref_lib.yoshida_direct(d, 1e-4, 1e-3, 20, order=ref_lib.ORDER_SIMD)
    for k in ("px", "py", "pz", "vx", "vy", "vz", "ax", "ay", "az"):
        np.testing.assert_array_equal(got[k], want[k], err_msg=k)


def test_engine_adaptive_update_equals_oracle_rule(ref_lib):
    """Engine::update with the adaptive time step: each step's dt is the
    oracle's clamp rule on the previous step's accelerations."""
    d = _state(256, 24)
    d["ax"], d["ay"], d["az"] = ref_lib.direct_forces_order(
        d["px"], d["py"], d["pz"], d["mass"], d["active"], 1e-4, ref_lib.ORDER_SIMD)
    eta, lo, hi, dt0 = 0.02, 1e-7, 5e-3, 1e-3
    got, steps, dt_last = ref_lib.ref_engine_update(d, 1e-4, 1e-3, 3.5e-3, 4, adaptive=True,
                                                    eta=eta, dt_min=lo, dt_max=hi, initial_dt=dt0)
    assert list(steps) == [3, 4, 3, 4]
    w = dict(d)
    dt = dt0
    for _ in range(int(steps.sum())):
        w = ref_lib.verlet_direct(w, 1e-4, dt, 1, order=ref_lib.ORDER_SIMD)
        w["active"] = d["active"]
        dt = ref_lib.adaptive_dt(w, 1e-4, eta, lo, hi)
    assert dt_last == dt
    for k in ("px", "py", "pz", "vx", "vy", "vz"):
        np.testing.assert_array_equal(got[k], w[k], err_msg=k)


@pytest.mark.parametrize("inactive", [0, 5])
def test_energy_tracker_restatement_identical(ref_lib, inactive):
    d = _state(700, 25, inactive)
    got = ref_lib.energy_tracker(d, 1e-4)
    want = ref_lib.ref_energy_tracker(d, 1e-4)
    assert got == want
    # the C# EnergyCalculator restatement sums in another order: close, not equal
    cs = ref_lib.energy(d, 1e-4)
    for k in ("ke", "pe", "e", "px", "lx", "comx", "m"):
        assert cs[k] == pytest.approx(want[k], rel=1e-12, abs=1e-18), k


@pytest.mark.parametrize("shell", [False, True])
def test_three_backend_orders_agree_within_ulps(oracle, shell):
    """CpuParallel, SIMD and single-thread (Newton's third law) orders: bit
    patterns differ, values agree to 1e-14 relative per body (the reference
    holds SIMD to scalar within 1e-12, SIMDParityTests.cs:62-100).  With
    the shell theorem on, the SIMD and single-thread backends run the
    CpuParallel arithmetic and the three are identical."""
    d = _state(800, 26, 9)
    rad = np.full(800, 0.02) if shell else None
    out = [oracle.direct_forces_order(d["px"], d["py"], d["pz"], d["mass"], d["active"], 1e-4, o,
                                      radius=rad, shell=shell) for o in range(3)]
    for o in (1, 2):
        err = rel_err(np.array(out[o]), np.array(out[0]))
        assert err.max() < 1e-14, (o, err.max())
        if shell:
            for x, y in zip(out[o], out[0]):
                np.testing.assert_array_equal(x, y)
    if not shell:
        assert not all(np.array_equal(x, y) for x, y in zip(out[2], out[0]))
        # inactive bodies get exactly zero in every order
        for o in range(3):
            assert np.all(out[o][0][~d["active"].astype(bool)] == 0.0)


def test_simd_order_lane_width_is_irrelevant(oracle):
    """n not a multiple of the lane count: the scalar tail uses the lanes'
    arithmetic, so the result equals a plain per-pair loop in that form."""
    d = _state(37, 27)
    got = oracle.direct_forces_order(d["px"], d["py"], d["pz"], d["mass"], d["active"], 1e-4, 1)
    px, py, pz, m = d["px"], d["py"], d["pz"], d["mass"]
    want = np.zeros((3, 37))
    for i in range(37):
        s = [0.0, 0.0, 0.0]
        for j in range(37):
            if j == i:
                continue
            dx, dy, dz = px[i] - px[j], py[i] - py[j], pz[i] - pz[j]
            inv = 1.0 / np.sqrt(dx * dx + dy * dy + dz * dz + 1e-8)
            f = m[j] * (inv * inv * inv)
            s = [s[0] - f * dx, s[1] - f * dy, s[2] - f * dz]
        want[:, i] = s
    for k in range(3):
        np.testing.assert_array_equal(got[k], want[k])
