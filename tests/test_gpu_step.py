"""Device-resident stepping, diagnostics, collisions and compaction on the
GPU against the oracle."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import bodies_dict
from nbody_b200 import (FLAG_ADAPTIVE_DT, FLAG_COLLISIONS, FLAG_SHELL_THEOREM, FLAG_YOSHIDA4,
                        MODE_BARNES_HUT, MODE_DIRECT_FP64, NBodyError, scenarios)
from nbody_b200.scenarios import Bodies
from nbody_b200 import _native as N

pytestmark = pytest.mark.gpu


def test_verlet_fp64_trajectory_bit_exact(engine, oracle):
    """K Verlet steps with the FP64 direct sum on the device reproduce the
    CPU SoAVerletIntegrator + CpuParallelBackend trajectory bit for bit."""
    b = scenarios.plummer(300, seed=0)
    b.active[::17] = 0
    engine.set_state(b)
    engine.step(50, 1e-3, 1e-4, MODE_DIRECT_FP64)
    got, ids = engine.get_state()
    want = oracle.verlet_direct(bodies_dict(b), 1e-4, 1e-3, 50)
    np.testing.assert_array_equal(ids, np.arange(300))
    for k in ("px", "py", "pz", "vx", "vy", "vz", "ax", "ay", "az"):
        np.testing.assert_array_equal(getattr(got, k), want[k], err_msg=k)


YOSHIDA_W1 = 1.0 / (2.0 - 1.2599210498948732)
YOSHIDA_W0 = -1.2599210498948732 / (2.0 - 1.2599210498948732)


def test_yoshida4_fp64_trajectory_bit_exact(engine, oracle):
    """Yoshida4 steps (three KDK sub-steps of w1 dt, w0 dt, w1 dt, as the
    reference's Engine::cpu_yoshida_substep composes them) with the FP64
    direct sum equal the oracle's Verlet sub-steps chained the same way, bit
    for bit, through the captured-graph path and the step-by-step path."""
    b = scenarios.plummer(300, seed=0)
    b.active[::17] = 0
    want = bodies_dict(b)
    for _ in range(20):
        for w in (YOSHIDA_W1, YOSHIDA_W0, YOSHIDA_W1):
            want = dict(oracle.verlet_direct(want | {"active": b.active}, 1e-4, w * 1e-3, 1),
                        active=b.active)
    for one_by_one in (False, True):
        engine.set_state(b)
        if one_by_one:
            for _ in range(20):
                engine.step(1, 1e-3, 1e-4, MODE_DIRECT_FP64 | FLAG_YOSHIDA4)
        else:
            engine.step(20, 1e-3, 1e-4, MODE_DIRECT_FP64 | FLAG_YOSHIDA4)
        got, _ = engine.get_state()
        for k in ("px", "py", "pz", "vx", "vy", "vz", "ax", "ay", "az"):
            np.testing.assert_array_equal(getattr(got, k), want[k], err_msg=(k, one_by_one))


def test_yoshida4_energy_error_is_fourth_order(engine):
    """Two bodies on an eccentric orbit (G = 1, total mass 1, separation 1 at
    apocentre, speeds 0.8 of circular): over 2 pi time units the energy error
    of Yoshida4 is far below Verlet's at the same dt, and shrinks about
    16-fold when dt halves (4th order; Verlet's shrinks 4-fold)."""
    def run(flags, dt):
        v = 0.4  # circular would be 0.5: v^2 / 0.5 = 0.5 / 1^2
        b = Bodies(px=np.array([0.5, -0.5]), py=np.zeros(2), pz=np.zeros(2),
                   vx=np.zeros(2), vy=np.array([v, -v]), vz=np.zeros(2),
                   mass=np.array([0.5, 0.5]), radius=np.zeros(2), active=np.ones(2, np.uint8))
        engine.set_state(b, old_acc=False)
        engine.step(1, 0.0, 1e-6, MODE_DIRECT_FP64)  # accelerations at the start
        e0 = engine.diagnostics(1e-6)["e"]
        steps = int(round(2 * np.pi / dt))
        errs = []
        for _ in range(steps):
            engine.step(1, dt, 1e-6, MODE_DIRECT_FP64 | flags)
            errs.append(abs(engine.diagnostics(1e-6)["e"] - e0) / abs(e0))
        return max(errs)

    ev = run(0, 0.02)
    ey = run(FLAG_YOSHIDA4, 0.02)
    ey2 = run(FLAG_YOSHIDA4, 0.01)
    assert ey < 0.05 * ev, (ey, ev)
    assert 8.0 < ey / ey2 < 32.0, (ey, ey2)


def _adaptive_dt_rule(st, active, eps, eta, lo, hi):
    """AdaptiveTimestep::compute_dt after a step: a_max over the active rows
    (NaN and zero rows skipped, as the reference's max loop skips them)."""
    a2 = st["ax"] * st["ax"] + st["ay"] * st["ay"] + st["az"] * st["az"]
    a2 = a2[active.astype(bool) & (a2 > 0)]
    amax = float(np.sqrt(a2.max())) if a2.size else 0.0
    if amax <= 0.0 or eps <= 0.0:
        return hi
    return min(max(eta * float(np.sqrt(eps / amax)), lo), hi)


def test_adaptive_dt_fp64_trajectory_bit_exact(engine, oracle):
    """FLAG_ADAPTIVE_DT: after every step dt becomes clamp(eta sqrt(eps /
    a_max), dt_min, dt_max); the dt sequence and the trajectory equal the
    oracle's Verlet steps under the same rule, bit for bit, whether the steps
    come one call at a time or in one call."""
    eps, eta, lo, hi = 1e-4, 0.02, 1e-6, 1e-3
    b = scenarios.plummer(300, seed=3)
    b.active[::13] = 0
    want, dt, dts = bodies_dict(b), 1e-4, []
    for _ in range(15):
        want = dict(oracle.verlet_direct(want | {"active": b.active}, eps, dt, 1), active=b.active)
        dt = _adaptive_dt_rule(want, b.active, eps, eta, lo, hi)
        dts.append(dt)
    assert len(set(dts)) > 1  # the rule moves dt
    engine.set_param(N.PARAM_ADAPTIVE_ETA, eta)
    engine.set_param(N.PARAM_ADAPTIVE_DT_MIN, lo)
    engine.set_param(N.PARAM_ADAPTIVE_DT_MAX, hi)
    try:
        for one_call in (False, True):
            engine.set_state(b)
            assert engine.adaptive_dt() == 0.0
            if one_call:
                engine.step(15, 1e-4, eps, MODE_DIRECT_FP64 | FLAG_ADAPTIVE_DT)
                assert engine.adaptive_dt() == dts[-1]
            else:
                got = []
                for _ in range(15):
                    engine.step(1, 1e-4, eps, MODE_DIRECT_FP64 | FLAG_ADAPTIVE_DT)
                    got.append(engine.adaptive_dt())
                assert got == dts
            st, _ = engine.get_state()
            for k in ("px", "py", "pz", "vx", "vy", "vz", "ax", "ay", "az"):
                np.testing.assert_array_equal(getattr(st, k), want[k], err_msg=(k, one_call))
    finally:
        engine.set_param(N.PARAM_ADAPTIVE_ETA, 0.01)
        engine.set_param(N.PARAM_ADAPTIVE_DT_MIN, 1e-8)
        engine.set_param(N.PARAM_ADAPTIVE_DT_MAX, 0.01)


def test_energy_drift_10k_steps_plummer_1000(engine, oracle):
    """The FP64 direct-sum workload (N=1000 Plummer, seed 0, eps 1e-4,
    dt 1e-3, 10k steps): the device run reproduces the CPU trajectory, so
    the energy drift is the CPU drift."""
    b = scenarios.plummer(1000, seed=0)
    engine.set_state(b, old_acc=False)
    e0 = engine.diagnostics(1e-4)["e"]
    engine.step(10_000, 1e-3, 1e-4, MODE_DIRECT_FP64)
    e1 = engine.diagnostics(1e-4)["e"]
    drift_gpu = (e1 - e0) / abs(e0)
    got, _ = engine.get_state()
    want = oracle.verlet_direct(bodies_dict(b), 1e-4, 1e-3, 10_000)
    want["active"] = b.active
    drift_cpu = (oracle.energy(want, 1e-4)["e"] - oracle.energy(bodies_dict(b), 1e-4)["e"]) / abs(e0)
    np.testing.assert_array_equal(got.px, want["px"])
    assert drift_gpu == pytest.approx(drift_cpu, rel=1e-6, abs=1e-12)


def test_diagnostics_match_oracle(engine, oracle):
    b = scenarios.plummer(5000, seed=4)
    b.active[::9] = 0
    engine.set_state(b)
    d = engine.diagnostics(1e-4, pe_mode=0)
    w = oracle.energy(bodies_dict(b), 1e-4)
    for k in ("ke", "pe", "e", "px", "py", "pz", "lx", "ly", "lz", "comx", "comy", "comz", "m"):
        assert d[k] == pytest.approx(w[k], rel=1e-11, abs=1e-14), k
    # tree potential (pe_mode 1) approximates the exact pair sum
    dt = engine.diagnostics(1e-4, pe_mode=1)
    assert dt["pe"] == pytest.approx(w["pe"], rel=1e-3)


def test_force_error_audit_matches_oracle(engine, oracle):
    b = scenarios.plummer(40_000, seed=6)
    engine.set_param(N.PARAM_THETA, 0.5)
    engine.set_state(b, old_acc=False)
    engine.step(1, 0.0, 1e-4, MODE_BARNES_HUT)  # dt = 0: forces at the initial positions
    mean, mx, rms = engine.force_error(0, 0, 1e-4)
    got, _ = engine.get_state()
    want = oracle.direct_forces(b.px, b.py, b.pz, b.mass, b.active, 1e-4)
    wm, wx, wr = oracle.force_error((got.ax, got.ay, got.az), want, b.active)
    assert mean == pytest.approx(wm, rel=1e-9) and rms == pytest.approx(wr, rel=1e-9)
    assert mx == pytest.approx(wx, rel=1e-9)
    assert rms < 1e-3


def _sample_rows(active, ns, seed):
    """The audit's sample: a SplitMix64-driven partial Fisher-Yates shuffle
    of the active rows in index order (the first ns of the shuffled list)."""
    m = (1 << 64) - 1
    x = seed
    cand = [int(i) for i in np.flatnonzero(active)]
    for k in range(ns):
        x = (x + 0x9E3779B97F4A7C15) & m
        z = x
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & m
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & m
        z ^= z >> 31
        j = k + z % (len(cand) - k)
        cand[k], cand[j] = cand[j], cand[k]
    return np.array(cand[:ns])


@pytest.mark.parametrize("inactive", [False, True])
def test_sampled_force_error_matches_oracle(engine, oracle, inactive):
    """A sampled audit (all rows active, and with inactive rows) draws the
    same bodies as the shuffle restated here and reports the oracle's
    statistics over them against the FP64 direct sum."""
    b = scenarios.plummer(30_000, seed=8)
    if inactive:
        b.active[::7] = 0
    engine.set_param(N.PARAM_THETA, 0.6)
    engine.set_state(b, old_acc=False)
    engine.step(1, 0.0, 1e-4, MODE_BARNES_HUT)
    got, _ = engine.get_state()
    for ns, seed in ((700, 3), (2500, 0x5EED)):
        mean, mx, rms = engine.force_error(ns, seed, 1e-4)
        t = _sample_rows(b.active, ns, seed)
        want = oracle.direct_forces_targets(b.px, b.py, b.pz, b.mass, b.active, 1e-4, t)
        wm, wx, wr = oracle.force_error((got.ax[t], got.ay[t], got.az[t]), want)
        assert mean == pytest.approx(wm, rel=1e-9) and rms == pytest.approx(wr, rel=1e-9)
        assert mx == pytest.approx(wx, rel=1e-9)


def test_merge_and_compaction_step_bit_exact(engine, oracle):
    """dt = 0 step with collisions: pairs, merges (sequential CPU-resolver
    semantics) and compaction equal the oracle's."""
    d = scenarios.collisional_disk(4000, seed=12, radius_scale=2500.0)
    engine.set_state(d, old_acc=False)
    engine.step(1, 0.0, 1e-4, MODE_BARNES_HUT | FLAG_SHELL_THEOREM | FLAG_COLLISIONS)
    c = engine.counters()
    got, ids = engine.get_state()
    lo, hi = oracle.broad_phase(d.px, d.py, d.pz, d.radius, d.active, d.collidable)
    out, nm = oracle.resolve_merges(bodies_dict(d), lo, hi)
    assert c[N.C_PAIRS] == len(lo) and c[N.C_MERGES] == nm and nm > 0
    dest, kept = oracle.compact_indices(out["active"], out["mass"])
    assert len(ids) == kept
    keep = np.nonzero(dest >= 0)[0]
    np.testing.assert_array_equal(ids, keep)
    for k in ("px", "py", "pz", "vx", "vy", "vz", "mass"):
        np.testing.assert_array_equal(getattr(got, k), out[k][keep], err_msg=k)
    # merged radii go through cbrt: CUDA's and the C library's agree to 1 ulp
    np.testing.assert_allclose(got.radius, out["radius"][keep], rtol=5e-16)


def test_merge_and_compaction_at_disk_size(engine, oracle):
    """The collisional-disk workload's size, 262,144 bodies + the central
    mass, radii scaled 100x (2,093 overlapping pairs at the start, so the
    64-per-frame and 2-per-body caps both bind): a dt = 0 step with
    collisions gives the oracle's pair count, merges (sequential
    CollisionResolver semantics) and compacted state, bit for bit (merged
    radii to cbrt's 1 ulp).  The oracle's broad phase is the all-pairs test,
    split over the host's threads."""
    d = scenarios.collisional_disk(262_144, seed=2, radius_scale=100.0)
    engine.set_state(d, old_acc=False)
    engine.step(1, 0.0, 1e-4, MODE_BARNES_HUT | FLAG_SHELL_THEOREM | FLAG_COLLISIONS)
    c = engine.counters()
    got, ids = engine.get_state()
    lo, hi = oracle.broad_phase(d.px, d.py, d.pz, d.radius, d.active, d.collidable,
                                nthreads=oracle.threads())
    out, nm = oracle.resolve_merges(bodies_dict(d), lo, hi)
    assert len(lo) > 1000 and nm == 64
    assert c[N.C_PAIRS] == len(lo) and c[N.C_MERGES] == nm
    dest, kept = oracle.compact_indices(out["active"], out["mass"])
    assert len(ids) == kept == d.n - nm
    keep = np.nonzero(dest >= 0)[0]
    np.testing.assert_array_equal(ids, keep)
    for k in ("px", "py", "pz", "vx", "vy", "vz", "mass"):
        np.testing.assert_array_equal(getattr(got, k), out[k][keep], err_msg=k)
    np.testing.assert_allclose(got.radius, out["radius"][keep], rtol=5e-16)


def test_yoshida4_with_merges_once_per_step(engine, oracle):
    """Yoshida4 with collisions: the three sub-steps run without collisions,
    then one broad phase, merge and compaction on the state at the end of the
    step (as the C# solver detects after its whole integrator step and the
    reference engine's GPU paths after the last sub-step).  Equal to the
    oracle's Yoshida4 step followed by its broad phase, merges and
    compaction; the merge count is that step's."""
    d = scenarios.collisional_disk(3000, seed=14, radius_scale=2500.0)
    d.ax, d.ay, d.az = oracle.direct_forces(d.px, d.py, d.pz, d.mass, d.active, 1e-4)
    b = bodies_dict(d)
    engine.set_param(N.PARAM_MAX_MERGES_FRAME, 64)
    engine.set_state(d, old_acc=True)
    dt = 2e-3
    engine.step(1, dt, 1e-4, MODE_DIRECT_FP64 | FLAG_YOSHIDA4 | FLAG_COLLISIONS)
    c = engine.counters()
    got, ids = engine.get_state()
    y = oracle.yoshida_direct(b, 1e-4, dt, 1)
    y["active"] = d.active.copy()
    y["radius"] = d.radius.copy()
    y["density"] = b["density"].copy()
    lo, hi = oracle.broad_phase(y["px"], y["py"], y["pz"], y["radius"], y["active"],
                                d.collidable)
    out, nm = oracle.resolve_merges(y, lo, hi)
    assert nm > 0 and c[N.C_MERGES] == nm and c[N.C_PAIRS] == len(lo)
    dest, kept = oracle.compact_indices(out["active"], out["mass"])
    keep = np.nonzero(dest >= 0)[0]
    np.testing.assert_array_equal(ids, keep)
    for k in ("px", "py", "pz", "vx", "vy", "vz", "mass"):
        np.testing.assert_array_equal(getattr(got, k), out[k][keep], err_msg=k)


def test_collisional_steps_conserve_mass_and_momentum(engine):
    d = scenarios.collisional_disk(20_000, seed=2, radius_scale=1500.0)
    engine.set_state(d, old_acc=False)
    p0 = engine.diagnostics(1e-4)
    engine.step(5, 1e-3, 1e-4, MODE_BARNES_HUT | FLAG_SHELL_THEOREM | FLAG_COLLISIONS)
    p1 = engine.diagnostics(1e-4)
    assert p1["m"] == pytest.approx(p0["m"], rel=1e-13)
    got, ids = engine.get_state()
    assert len(ids) <= 20_001 and np.all(np.diff(ids) > 0)


def _collisional_run(d, flags, dt, steps, one_by_one):
    from nbody_b200 import Engine

    with Engine(1 << 21, device=0) as e:  # room for the pairs of the first steps
        e.set_state(d, old_acc=False)
        if one_by_one:
            for _ in range(steps):
                e.step(1, dt, 1e-4, flags)
        else:
            e.step(steps, dt, 1e-4, flags)
        st, ids = e.get_state()
        return st, ids, e.counters()


@pytest.mark.parametrize("n, scale, dt, steps, yoshida", [
    (20_000, 1500.0, 1e-3, 5, False),     # merges in every step, odd step count
    (262_145, 100.0, 0.0, 3, False),      # 2,093 pairs in the first step: the large pair sort
    (20_000, 1500.0, 1e-3, 4, True),      # Yoshida4 sub-steps, collisions after the last
])
def test_captured_collisional_steps_equal_single_steps(n, scale, dt, steps, yoshida):
    """Multi-step collisional calls replay two captured steps that keep every
    count on the device (the merge block sorts the pairs itself; compaction
    hands the row count to the next step): the state, row ids and the last
    step's pair and merge counts equal those of one nb_step(1) per step, the
    path pinned to the oracle above, bit for bit."""
    d = scenarios.collisional_disk(n - 1, seed=2, radius_scale=scale)
    flags = MODE_BARNES_HUT | FLAG_SHELL_THEOREM | FLAG_COLLISIONS
    if yoshida:
        flags |= FLAG_YOSHIDA4
    a, ida, ca = _collisional_run(d, flags, dt, steps, one_by_one=False)
    b, idb, cb = _collisional_run(d, flags, dt, steps, one_by_one=True)
    assert len(ida) < n  # bodies merged
    np.testing.assert_array_equal(ida, idb)
    for k in ("px", "py", "pz", "vx", "vy", "vz", "ax", "ay", "az", "mass", "radius"):
        np.testing.assert_array_equal(getattr(a, k), getattr(b, k), err_msg=k)
    assert ca[N.C_PAIRS] == cb[N.C_PAIRS] and ca[N.C_MERGES] == cb[N.C_MERGES]


def test_step_before_state_is_an_error():
    from nbody_b200 import Engine

    with Engine(1024) as e:
        with pytest.raises(NBodyError) as err:
            e.step(1, 1e-3, 1e-4, MODE_BARNES_HUT)
        assert err.value.status == N.NB_ERR_STATE
