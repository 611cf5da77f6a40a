"""The `celestial_*` compatibility layer on the GPU, against the oracle and
the reference's own Engine (oracle/_ref): the same trajectories bit for bit
as the reference's CPU brute force (Verlet and Yoshida4 steps, the frame
accumulator with the adaptive time step), energy and momentum drift as
EnergyTracker defines them, counts, refused collision modes and the
lifecycle rules."""
from __future__ import annotations

import numpy as np
import pytest

import compat_api as A
from conftest import bodies_dict
from nbody_b200 import scenarios

pytestmark = pytest.mark.gpu

W1 = 1.0 / (2.0 - 1.2599210498948732)
W0 = -1.2599210498948732 / (2.0 - 1.2599210498948732)
EPS = 1e-4


@pytest.fixture
def lib():
    from nbody_b200 import _native as N

    lib = A.bind(N.lib)
    assert lib.celestial_init(512) == 0, lib.celestial_get_last_error_message()
    # settings outlive shutdown/init, as the reference's global config does:
    # start every test from the defaults
    lib.celestial_set_integrator(0)
    lib.celestial_set_compute_mode(2)
    lib.celestial_set_collision_mode(0)
    lib.celestial_set_adaptive_timestep(0, 0.01, 1e-8, 0.01, 0.001)
    yield lib
    lib.celestial_shutdown()


def _upload(lib, b):
    arrs = [np.ascontiguousarray(getattr(b, k), np.float64)
            for k in ("px", "py", "pz", "vx", "vy", "vz", "ax", "ay", "az", "mass", "radius")]
    act = np.ascontiguousarray(b.active, np.uint8)
    lib.celestial_set_particles(*(a.ctypes.data for a in arrs), act.ctypes.data, b.n)
    return arrs, act


def _download(lib, n):
    out = {k: np.empty(n) for k in ("px", "py", "pz", "vx", "vy", "vz", "ax", "ay", "az")}
    lib.celestial_get_positions(out["px"].ctypes.data, out["py"].ctypes.data,
                                out["pz"].ctypes.data, n)
    lib.celestial_get_velocities(out["vx"].ctypes.data, out["vy"].ctypes.data,
                                 out["vz"].ctypes.data, n)
    lib.celestial_get_accelerations(out["ax"].ctypes.data, out["ay"].ctypes.data,
                                    out["az"].ctypes.data, n)
    return out


def _chain(oracle, b, dts):
    """Verlet steps of the given dts with the reference engine's CPU
    brute-force arithmetic (the SIMD-backend order)."""
    s = bodies_dict(b)
    for dt in dts:
        s = dict(oracle.verlet_direct(s | {"active": b.active}, EPS, dt, 1,
                                      order=oracle.ORDER_SIMD), active=b.active)
    return s


def _assert_same(got, want, what):
    for k in ("px", "py", "pz", "vx", "vy", "vz", "ax", "ay", "az"):
        np.testing.assert_array_equal(got[k], want[k], err_msg=(what, k))


def test_compat_verlet_and_yoshida_bit_exact(lib, oracle):
    b = scenarios.plummer(300, seed=0)
    b.active[::17] = 0
    _upload(lib, b)
    assert lib.celestial_get_particle_count() == 300
    assert lib.celestial_get_active_particle_count() == int(b.active.sum())
    for _ in range(10):
        lib.celestial_step(1e-3, EPS)
    _assert_same(_download(lib, 300), _chain(oracle, b, [1e-3] * 10), "verlet")
    assert lib.celestial_get_last_gpu_time_ms() >= 0.0
    # Yoshida4: three KDK sub-steps of w1 dt, w0 dt, w1 dt per step
    lib.celestial_set_integrator(1)
    assert lib.celestial_get_integrator() == 1
    _upload(lib, b)
    for _ in range(5):
        lib.celestial_step(1e-3, EPS)
    _assert_same(_download(lib, 300), _chain(oracle, b, [W1 * 1e-3, W0 * 1e-3, W1 * 1e-3] * 5),
                 "yoshida4")
    assert lib.celestial_get_last_error_message() == b""


def test_compat_update_with_adaptive_dt(lib, oracle):
    """celestial_update: steps of the init-time dt (0.001) fit in the frame
    time, each taking the adaptive dt, which the rule updates after every
    step (AdaptiveTimestep)."""
    b = scenarios.plummer(300, seed=5)
    eta, lo, hi, dt0 = 0.02, 1e-6, 1e-3, 2e-4
    lib.celestial_set_adaptive_timestep(1, eta, lo, hi, dt0)
    assert lib.celestial_is_adaptive_dt_enabled() == 1
    assert lib.celestial_get_adaptive_dt() == dt0
    _upload(lib, b)
    assert lib.celestial_update(0.0035) == 3  # 3 whole steps of 0.001 in the frame
    s, dt, dts = bodies_dict(b), dt0, []
    for _ in range(3):
        dts.append(dt)
        s = dict(oracle.verlet_direct(s | {"active": b.active}, EPS, dt, 1,
                                      order=oracle.ORDER_SIMD), active=b.active)
        a2 = s["ax"] * s["ax"] + s["ay"] * s["ay"] + s["az"] * s["az"]
        amax = float(np.sqrt(a2[b.active.astype(bool) & (a2 > 0)].max()))
        dt = min(max(eta * float(np.sqrt(EPS / amax)), lo), hi)
    _assert_same(_download(lib, 300), s, "adaptive")
    assert lib.celestial_get_adaptive_dt() == dt
    assert len(set(dts)) > 1
    # the accumulator keeps the remainder: 0.0005 + 0.0006 makes one more step
    assert lib.celestial_update(0.0006) == 1


@pytest.mark.parametrize("integrator", [0, 1])
def test_compat_bit_exact_with_the_reference_engine(lib, ref_lib, integrator):
    """CPU_BruteForce through the compatibility layer against the reference's
    own Engine (engine.cpp compiled into oracle/_ref) on the same input:
    identical trajectories, Leapfrog_KDK and Yoshida4."""
    b = scenarios.plummer(400, seed=31)
    b.active[7::29] = 0
    d = bodies_dict(b)
    d["ax"], d["ay"], d["az"] = ref_lib.direct_forces_order(
        b.px, b.py, b.pz, b.mass, b.active, EPS, ref_lib.ORDER_SIMD)
    lib.celestial_set_compute_mode(0)
    lib.celestial_set_integrator(integrator)
    arrs = [np.ascontiguousarray(d[k], np.float64)
            for k in ("px", "py", "pz", "vx", "vy", "vz", "ax", "ay", "az", "mass", "radius")]
    act = np.ascontiguousarray(b.active, np.uint8)
    lib.celestial_set_particles(*(a.ctypes.data for a in arrs), act.ctypes.data, b.n)
    for _ in range(12):
        lib.celestial_step(1e-3, EPS)
    want = ref_lib.ref_engine_steps(d, EPS, 1e-3, 12, compute_mode=0, integrator=integrator)
    _assert_same(_download(lib, 400), want, f"reference engine, integrator {integrator}")


def test_compat_adaptive_update_bit_exact_with_the_reference_engine(lib, ref_lib):
    """celestial_update with the adaptive time step against the reference's
    Engine::update on the same input: the same step counts, final dt and
    trajectory."""
    b = scenarios.plummer(300, seed=32)
    d = bodies_dict(b)
    d["ax"], d["ay"], d["az"] = ref_lib.direct_forces_order(
        b.px, b.py, b.pz, b.mass, b.active, EPS, ref_lib.ORDER_SIMD)
    eta, lo, hi, dt0 = 0.02, 1e-7, 5e-3, 1e-3
    lib.celestial_set_compute_mode(0)
    lib.celestial_set_adaptive_timestep(1, eta, lo, hi, dt0)
    arrs = [np.ascontiguousarray(d[k], np.float64)
            for k in ("px", "py", "pz", "vx", "vy", "vz", "ax", "ay", "az", "mass", "radius")]
    act = np.ascontiguousarray(b.active, np.uint8)
    lib.celestial_set_particles(*(a.ctypes.data for a in arrs), act.ctypes.data, b.n)
    got_steps = [lib.celestial_update(3.5e-3) for _ in range(4)]
    want, steps, dt_last = ref_lib.ref_engine_update(d, EPS, 1e-3, 3.5e-3, 4, adaptive=True,
                                                     eta=eta, dt_min=lo, dt_max=hi,
                                                     initial_dt=dt0)
    assert got_steps == list(steps)
    assert lib.celestial_get_adaptive_dt() == dt_last
    got = _download(lib, 300)
    for k in ("px", "py", "pz", "vx", "vy", "vz"):
        np.testing.assert_array_equal(got[k], want[k], err_msg=k)


def test_compat_new_scene_restarts_the_energy_tracker(lib):
    """celestial_set_particles resets the drift bookkeeping, as the
    reference's Engine::set_particles does (engine.cpp:195): the first
    snapshot of a new scene is its own baseline."""
    a = scenarios.plummer(200, seed=33)
    _upload(lib, a)
    lib.celestial_compute_forces(EPS)
    lib.celestial_compute_energy_snapshot()
    for _ in range(5):
        lib.celestial_step(1e-3, EPS)
    lib.celestial_compute_energy_snapshot()
    assert lib.celestial_get_accumulated_error() > 0.0
    b = scenarios.plummer(250, seed=34)
    _upload(lib, b)
    lib.celestial_compute_forces(EPS)
    lib.celestial_compute_energy_snapshot()
    assert lib.celestial_get_energy_drift() == 0.0
    assert lib.celestial_get_momentum_drift() == 0.0
    assert lib.celestial_get_angular_momentum_drift() == 0.0
    assert lib.celestial_get_accumulated_error() == 0.0


def test_compat_getters_copy_count_rows(lib):
    """The getters fill `count` rows; fewer than the state holds is fine."""
    b = scenarios.plummer(128, seed=35)
    _upload(lib, b)
    full = _download(lib, 128)
    part = _download(lib, 50)
    for k in ("px", "vy", "az"):
        np.testing.assert_array_equal(part[k], full[k][:50])


def test_compat_energy_drift_as_energy_tracker(lib, oracle):
    b = scenarios.plummer(200, seed=2)
    _upload(lib, b)
    lib.celestial_compute_forces(EPS)
    lib.celestial_compute_energy_snapshot()
    assert lib.celestial_get_energy_drift() == 0.0
    s0 = _download(lib, 200) | {"mass": b.mass, "active": b.active}
    for _ in range(20):
        lib.celestial_step(1e-3, EPS)
    lib.celestial_compute_energy_snapshot()
    s1 = _download(lib, 200) | {"mass": b.mass, "active": b.active}
    e0, e1 = oracle.energy(s0, EPS), oracle.energy(s1, EPS)
    want = (e1["e"] - e0["e"]) / abs(e0["e"])
    # the device and oracle energies agree to ~1e-11 relative (summation
    # order), so a drift of ~1e-8 agrees to ~2e-11 absolute
    assert lib.celestial_get_energy_drift() == pytest.approx(want, rel=1e-9, abs=5e-11)
    dp = np.sqrt(sum((e1[k] - e0[k]) ** 2 for k in ("px", "py", "pz")))
    assert lib.celestial_get_momentum_drift() == pytest.approx(dp, rel=1e-6, abs=1e-13)
    assert lib.celestial_get_accumulated_error() == pytest.approx(abs(want), rel=1e-9, abs=5e-11)


def test_compat_modes_collisions_and_lifecycle(lib):
    assert lib.celestial_init(16) == -7  # AlreadyInitialized
    lib.celestial_set_collision_mode(1)  # Elastic: refused
    assert b"not supported" in lib.celestial_get_last_error_message()
    lib.celestial_set_collision_mode(3)  # Merge
    assert lib.celestial_get_last_error_message() == b""
    lib.celestial_set_collision_mode(0)
    b = scenarios.plummer(400, seed=9)
    _upload(lib, b)
    for mode in (1, 3):  # the Barnes-Hut modes run and keep every body
        lib.celestial_set_compute_mode(mode)
        lib.celestial_step(1e-4, EPS)
        assert lib.celestial_get_last_error_message() == b"", mode
        got = _download(lib, 400)
        assert np.all(np.isfinite(got["ax"]))
    assert lib.celestial_get_last_tree_traverse_ms() > 0.0
    lib.celestial_shutdown()
    assert lib.celestial_get_particle_count() == 0
    assert lib.celestial_init(64) == 0
