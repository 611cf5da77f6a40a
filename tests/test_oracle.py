"""The oracle restatement against the reference's own CPU code (oracle/_ref)
and against the reference's known-answer tests.  CPU only."""
from __future__ import annotations

import numpy as np
import pytest

from helpers import ref_canonical, rel_err, trig_bodies
from nbody_b200 import scenarios


def _clusters(n, seed):
    """Two Gaussian clusters (cf. engine/tests/test_phase18_19.cpp:38-67)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    c = rng.choice(2, n)
    centers = np.array([[-3.0, 0.0, 0.0], [3.0, 1.0, -1.0]])
    p = centers[c] + rng.standard_normal((n, 3))
    m = rng.uniform(0.5, 1.5, n)
    return p[:, 0].copy(), p[:, 1].copy(), p[:, 2].copy(), m


# ---- restatement == reference code -------------------------------------

def test_octree_identical_to_reference(ref_lib):
    b = scenarios.plummer(3000, seed=11)
    b.active[::17] = 0
    a = ref_lib.octree(b.px, b.py, b.pz, b.mass, b.active)
    r = ref_lib.ref_octree(b.px, b.py, b.pz, b.mass, b.active)
    for k in ("center", "mass", "com", "children", "body", "leaf"):
        np.testing.assert_array_equal(a[k], r[k], err_msg=k)


@pytest.mark.parametrize("theta", [0.0, 0.3, 0.5, 1.0])
def test_bh_forces_identical_to_reference(ref_lib, theta):
    b = scenarios.plummer(2000, seed=12)
    b.active[5::23] = 0
    mine = ref_lib.bh_forces(b.px, b.py, b.pz, b.mass, b.active, 1e-4, theta)
    (ref, _, _) = ref_lib.ref_bh_forces(b.px, b.py, b.pz, b.mass, b.active, 1e-4, theta)
    for x, y in zip(mine, ref):
        np.testing.assert_array_equal(x, y)


def test_bh_parallel_reference_matches_serial(ref_lib):
    b = scenarios.plummer(4000, seed=13)
    (s, _, _) = ref_lib.ref_bh_forces(b.px, b.py, b.pz, b.mass, b.active, 1e-4, 0.5, False)
    (p, _, _) = ref_lib.ref_bh_forces(b.px, b.py, b.pz, b.mass, b.active, 1e-4, 0.5, True, 4)
    for x, y in zip(s, p):
        np.testing.assert_array_equal(x, y)


def test_morton_matches_reference_morton_from_unit(ref_lib):
    rng = np.random.Generator(np.random.PCG64(3))
    u = rng.random((500, 3))
    u[0] = 0.0
    u[1] = 1.0
    u[2] = [0.5, 1.0 - 1e-16, 1e-300]
    # bbox exactly [0,1]^3 so the oracle's normalisation is the identity
    px, py, pz = u[:, 0].copy(), u[:, 1].copy(), u[:, 2].copy()
    keys, _ = ref_lib.morton_aabb(px, py, pz, np.ones(500, np.uint8))
    want = [ref_lib.ref().ref_morton_from_unit(*row) for row in u]
    np.testing.assert_array_equal(keys, np.array(want, np.uint64))


def test_compaction_matches_reference(ref_lib):
    rng = np.random.Generator(np.random.PCG64(4))
    n = 5000
    act = (rng.random(n) > 0.25).astype(np.uint8)
    mass = rng.uniform(0.5, 2.0, n)
    dest, kept = ref_lib.compact_indices(act, mass)
    arrs = [rng.standard_normal(n) for _ in range(6)]
    c = [a.copy() for a in arrs]
    mc, ac = mass.copy(), act.copy()
    p = lambda a: a.ctypes.data  # noqa: E731
    k = ref_lib.ref().ref_compact(n, *(p(x) for x in c), p(mc), p(ac))
    assert k == kept
    sel = dest >= 0
    for a, r in zip(arrs, c):
        out = np.empty(kept)
        out[dest[sel]] = a[sel]
        np.testing.assert_array_equal(out, r[:kept])


def test_merges_match_reference(ref_lib):
    d = scenarios.collisional_disk(3000, seed=9, radius_scale=2500.0)
    lo, hi = ref_lib.broad_phase(d.px, d.py, d.pz, d.radius, d.active, d.collidable)
    assert len(lo) > 64
    bd = {k: getattr(d, k) for k in ("px", "py", "pz", "vx", "vy", "vz", "mass", "radius",
                                      "density", "active")}
    for kw in ({}, {"max_frame": 10000, "max_body": 1}, {"density_merge": 0}):
        a, ka = ref_lib.resolve_merges(bd, lo, hi, **kw)
        r, kr = ref_lib.ref_resolve_merges(bd, lo, hi, **kw)
        assert ka == kr
        for k in a:
            np.testing.assert_array_equal(a[k], r[k], err_msg=k)


# ---- known-answer tests of the reference, on the restatement -----------

def test_two_body_unit_acceleration(oracle):
    """engine/tests/test_gravity.cpp:16-45."""
    px, py, pz = np.array([-0.5, 0.5]), np.zeros(2), np.zeros(2)
    m = np.ones(2)
    act = np.ones(2, np.uint8)
    ax, ay, az = oracle.direct_forces(px, py, pz, m, act, 0.0)
    assert ax[0] == pytest.approx(1.0, abs=1e-10) and ax[1] == pytest.approx(-1.0, abs=1e-10)
    bx, _, _ = oracle.bh_forces(px, py, pz, m, act, 0.0, 0.0)
    np.testing.assert_allclose(bx, ax, atol=1e-10)


def test_inactive_bodies_get_zero(oracle):
    """engine/tests/test_gravity.cpp:108-130."""
    px = np.array([0.0, 1.0, 2.0])
    z = np.zeros(3)
    act = np.array([1, 0, 1], np.uint8)
    ax, ay, az = oracle.direct_forces(px, z, z, np.ones(3), act, 0.0)
    assert ax[1] == 0.0 and ay[1] == 0.0 and az[1] == 0.0
    assert ax[0] == pytest.approx(0.25)


def test_octants_and_tree_mass(oracle):
    """engine/tests/test_octree.cpp:24-115: x -> bit 0, y -> bit 1, z -> bit 2;
    root mass and COM."""
    s = np.array([-1.0, 1.0])
    pts = np.array([[x, y, z] for z in s for y in s for x in s])
    t = oracle.octree(pts[:, 0], pts[:, 1], pts[:, 2], np.ones(8), np.ones(8, np.uint8))
    assert t["mass"][0] == 8.0
    for octant in range(8):
        c = t["children"][0][octant]
        assert c >= 0 and t["leaf"][c] and t["body"][c] == octant
    i = np.arange(50, dtype=np.float64)
    t = oracle.octree(i * 0.1, i * 0.2, i * 0.05, np.ones(50), np.ones(50, np.uint8))
    assert t["mass"][0] == 50.0


def test_bh_vs_exact_trig_fixture(oracle):
    """engine/tests/test_gravity.cpp:67-105: theta 0.5 within 5% per x
    component of the solver run with theta = 0 (which the solver clamps to
    0.2, barnes_hut_solver.cpp:16)."""
    px, py, pz, m = trig_bodies(20)
    act = np.ones(20, np.uint8)
    ex = oracle.bh_forces(px, py, pz, m, act, 1e-4, 0.0)
    bh = oracle.bh_forces(px, py, pz, m, act, 1e-4, 0.5)
    big = np.abs(ex[0]) > 1e-10
    err = np.abs((bh[0][big] - ex[0][big]) / ex[0][big])
    # The reference's own solver gives 0.0814 on body 17 of this fixture, so
    # the gtest's 5% bound does not hold for the reference itself; the
    # restatement reproduces that value exactly.
    assert err.max() == pytest.approx(0.08138851332462206, rel=1e-12)
    assert np.median(err) < 0.05


def test_bh_rms_below_one_percent_and_monotone(oracle):
    """engine/tests/test_phase18_19.cpp:74-205."""
    px, py, pz, m = _clusters(128, 12345)
    act = np.ones(128, np.uint8)
    ex = oracle.direct_forces(px, py, pz, m, act, 1e-3)
    prev = np.inf
    for th in (0.8, 0.5, 0.3):
        bh = oracle.bh_forces(px, py, pz, m, act, 1e-3, th)
        rms = np.sqrt(np.mean(rel_err(bh, ex) ** 2))
        if th == 0.5:
            assert rms < 0.01
        assert rms <= prev + 1e-12
        prev = rms


def test_theta_zero_clamps_to_point_two(oracle):
    """BarnesHutAccuracyTests.cs:164-186 (theta < 0.2 behaves as 0.2)."""
    b = scenarios.plummer(400, seed=2)
    a0 = oracle.bh_forces(b.px, b.py, b.pz, b.mass, b.active, 1e-4, 0.0)
    a2 = oracle.bh_forces(b.px, b.py, b.pz, b.mass, b.active, 1e-4, 0.2)
    for x, y in zip(a0, a2):
        np.testing.assert_array_equal(x, y)


def test_shell_theorem_inside_outside(oracle):
    """GravityTests.cs:107-195: linear interior field, continuity at R."""
    R = 1.0
    for d, inside in ((0.5, True), (0.999999, True), (1.000001, False), (2.0, False)):
        px = np.array([0.0, d])
        z = np.zeros(2)
        rad = np.array([R, 0.0])
        ax, _, _ = oracle.direct_forces(px, z, z, np.array([1.0, 1e-12]), np.ones(2, np.uint8),
                                        1e-4, radius=rad, shell=True)
        want = -d / (R * R + 1e-8) ** 1.5 if inside else -d / (d * d + 1e-8) ** 1.5
        assert ax[1] == pytest.approx(want, rel=1e-12)


def test_two_body_verlet_drift(oracle):
    """SoAStabilityTests.cs:68-132: circular two-body orbit, dt 1e-3, 10k
    steps, relative energy drift < 1e-4."""
    v = np.sqrt(0.5 / 1.0) / 1.0  # equal unit masses at separation 1
    b = dict(px=np.array([-0.5, 0.5]), py=np.zeros(2), pz=np.zeros(2),
             vx=np.zeros(2), vy=np.array([-v / np.sqrt(2) * 1.0, v / np.sqrt(2)]) * np.sqrt(2) / 2,
             vz=np.zeros(2), ax=np.zeros(2), ay=np.zeros(2), az=np.zeros(2),
             mass=np.ones(2), active=np.ones(2, np.uint8))
    e0 = oracle.energy(b, 1e-4)["e"]
    out = oracle.verlet_direct(b, 1e-4, 1e-3, 10000)
    out["active"] = b["active"]
    e1 = oracle.energy(out, 1e-4)["e"]
    assert abs((e1 - e0) / e0) < 1e-4


def test_yoshida4_composition_is_fourth_order(oracle):
    """The Yoshida4 step the GPU tests compare against (three oracle Verlet
    sub-steps of w1 dt, w0 dt, w1 dt, yoshida.hpp:19-24): on an eccentric
    two-body orbit its energy error is far below Verlet's and falls 16-fold
    per halving of dt (Verlet's 4-fold)."""
    w1 = 1.0 / (2.0 - 1.2599210498948732)
    w0 = -1.2599210498948732 / (2.0 - 1.2599210498948732)
    b0 = dict(px=np.array([0.5, -0.5]), py=np.zeros(2), pz=np.zeros(2), vx=np.zeros(2),
              vy=np.array([0.4, -0.4]), vz=np.zeros(2), ax=np.zeros(2), ay=np.zeros(2),
              az=np.zeros(2), mass=np.array([0.5, 0.5]), active=np.ones(2, np.uint8))
    eps = 1e-6

    def err(yoshida, dt):
        s = dict(oracle.verlet_direct(b0, eps, 0.0, 1), active=b0["active"])  # a at t = 0
        e0 = oracle.energy(s, eps)["e"]
        worst = 0.0
        for _ in range(int(round(2 * np.pi / dt))):
            for h in ((w1 * dt, w0 * dt, w1 * dt) if yoshida else (dt,)):
                s = dict(oracle.verlet_direct(s, eps, h, 1), active=b0["active"])
            worst = max(worst, abs(oracle.energy(s, eps)["e"] - e0) / abs(e0))
        return worst

    v1, v2 = err(False, 0.02), err(False, 0.01)
    y1, y2 = err(True, 0.02), err(True, 0.01)
    assert y1 < 0.05 * v1
    assert 3.0 < v1 / v2 < 5.0 and 8.0 < y1 / y2 < 32.0, (v1 / v2, y1 / y2)


def test_yoshida_and_adaptive_restatements(oracle):
    """or_yoshida_direct (Engine::cpu_yoshida_substep x 3) equals three
    chained Verlet sub-steps bit for bit, and or_adaptive_dt applies the
    AdaptiveTimestep rule to the largest active |a| (clamped both ways)."""
    b = scenarios.plummer(120, seed=4)
    b.active[::9] = 0
    d = {k: v for k, v in b.__dict__.items()}
    w1 = 1.0 / (2.0 - 1.2599210498948732)
    w0 = -1.2599210498948732 / (2.0 - 1.2599210498948732)
    want = d
    for _ in range(4):
        for w in (w1, w0, w1):
            want = dict(oracle.verlet_direct(want, 1e-4, w * 1e-3, 1), active=b.active)
    got = oracle.yoshida_direct(d, 1e-4, 1e-3, 4)
    for k in ("px", "py", "pz", "vx", "vy", "vz", "ax", "ay", "az"):
        np.testing.assert_array_equal(got[k], want[k], err_msg=k)
    s = dict(got, active=b.active)
    act = b.active.astype(bool)
    a2 = s["ax"] * s["ax"] + s["ay"] * s["ay"] + s["az"] * s["az"]
    amax = np.sqrt(a2[act].max())
    assert oracle.adaptive_dt(s, 1e-4, 0.02, 1e-9, 1.0) == 0.02 * np.sqrt(1e-4 / amax)
    assert oracle.adaptive_dt(s, 1e-4, 0.02, 1e-9, 1e-7) == 1e-7     # ceiling
    assert oracle.adaptive_dt(s, 1e-4, 0.02, 1.0, 2.0) == 1.0        # floor
    assert oracle.adaptive_dt(s, 0.0, 0.02, 1e-9, 3e-3) == 3e-3      # no softening: dt_max


def test_stable_sort_semantics(oracle):
    rng = np.random.Generator(np.random.PCG64(1))
    keys = rng.integers(0, 50, 20000).astype(np.uint64) << np.uint64(40)
    vals = np.arange(20000, dtype=np.int32)
    k, v = oracle.stable_sort(keys, vals)
    order = np.argsort(keys, kind="stable")
    np.testing.assert_array_equal(k, keys[order])
    np.testing.assert_array_equal(v, vals[order])


def test_force_error_metric(oracle):
    a = (np.array([1.0, 0.0]), np.zeros(2), np.zeros(2))
    r = (np.array([1.1, 0.0]), np.zeros(2), np.zeros(2))
    mean, mx, rms = oracle.force_error(a, r)
    assert mx == pytest.approx(0.1 / 1.1) and mean == pytest.approx(0.1 / 1.1)


def test_canonical_form_of_reference_tree(ref_lib):
    """Sanity of the canonical form used by the GPU topology test: every
    body appears in exactly one depth-0 entry."""
    px, py, pz, m = trig_bodies(100)
    t = ref_lib.ref_octree(px, py, pz, m, np.ones(100, np.uint8))
    c = ref_canonical(t)
    roots = [e for e in c if e[0] == 0]
    assert len(roots) == 1 and len(roots[0][4]) == 100
