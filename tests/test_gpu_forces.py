"""Forces on the GPU against the oracle and the reference's own code.

Tolerances:
  * NB_MODE_DIRECT_FP64: bit-exact with the CpuParallelBackend restatement.
  * NB_MODE_DIRECT (FP32 pairs, FP64-differenced coordinates, compensated
    sums): per-body relative error vs FP64 rms < 2e-6, max < 1e-4.
  * NB_MODE_BARNES_HUT_REF (FP64, reference MAC): per-body relative error vs
    the reference BarnesHutSolver max < 1e-9.
  * NB_MODE_BARNES_HUT, theta 0.5, monopole + quadrupole: rms relative force
    error vs the FP64 direct sum < 1e-3 (the engine's force-error target).
"""
from __future__ import annotations

import numpy as np
import pytest

from helpers import rel_err, trig_bodies
from nbody_b200 import (FLAG_NO_QUADRUPOLE, FLAG_SHELL_THEOREM, MODE_BARNES_HUT,
                        MODE_BARNES_HUT_REF, MODE_DIRECT, MODE_DIRECT_FP64, NBodyError,
                        scenarios)
from nbody_b200 import _native as N

pytestmark = pytest.mark.gpu


def _forces(engine, b, eps, flags, theta=0.5):
    engine.set_param(N.PARAM_THETA, float(theta))
    return engine.compute_forces(b.px, b.py, b.pz, b.mass, b.active, eps, flags, radius=b.radius)


def test_direct_fp64_bit_exact_plummer_1000(engine, oracle):
    b = scenarios.plummer(1000, seed=0)  # the FP64 direct-sum workload, seed 0
    got = _forces(engine, b, 1e-4, MODE_DIRECT_FP64)
    want = oracle.direct_forces(b.px, b.py, b.pz, b.mass, b.active, 1e-4)
    for g, w in zip(got, want):
        np.testing.assert_array_equal(g, w)


def test_direct_fp64_bit_exact_inactive_and_shell(engine, oracle):
    d = scenarios.collisional_disk(700, seed=3, radius_scale=3000.0)
    d.active[::5] = 0
    got = _forces(engine, d, 1e-4, MODE_DIRECT_FP64 | FLAG_SHELL_THEOREM)
    want = oracle.direct_forces(d.px, d.py, d.pz, d.mass, d.active, 1e-4, radius=d.radius,
                                shell=True)
    for g, w in zip(got, want):
        np.testing.assert_array_equal(g, w)
    assert np.all(got[0][d.active == 0] == 0.0)


@pytest.mark.parametrize("order", [1, 2])
@pytest.mark.parametrize("n,inactive", [(1000, 0), (1531, 13)])
def test_direct_fp64_backend_orders_bit_exact(engine, oracle, order, n, inactive):
    """NB_FLAG_ORDER_SIMD / NB_FLAG_ORDER_PAIRWISE give the bits of the SIMD
    backend (and the native engine's CPU brute force) and of the
    single-thread Newton's-third-law backend."""
    b = scenarios.plummer(n, seed=40 + order)
    if inactive:
        b.active[::inactive] = 0
    flag = N.FLAG_ORDER_SIMD if order == 1 else N.FLAG_ORDER_PAIRWISE
    got = _forces(engine, b, 1e-4, MODE_DIRECT_FP64 | flag)
    want = oracle.direct_forces_order(b.px, b.py, b.pz, b.mass, b.active, 1e-4, order)
    for g, w in zip(got, want):
        np.testing.assert_array_equal(g, w)


def test_direct_fp64_engine_order_equals_reference_engine(engine, ref_lib):
    """The SIMD-order flag against the reference's own Engine CPU brute force
    (oracle/_ref) on the same input: identical accelerations."""
    b = scenarios.plummer(900, seed=44)
    b.active[2::31] = 0
    got = _forces(engine, b, 1e-4, MODE_DIRECT_FP64 | N.FLAG_ORDER_SIMD)
    d = {k: getattr(b, k) for k in ("px", "py", "pz", "vx", "vy", "vz", "ax", "ay", "az",
                                     "mass", "active")}
    d["radius"] = None
    want = ref_lib.ref_engine_steps(d, 1e-4, 0.0, 1)
    for g, k in zip(got, ("ax", "ay", "az")):
        np.testing.assert_array_equal(g, want[k])


def test_direct_fp64_orders_with_shell_theorem_are_cpuparallel(engine, oracle):
    d = scenarios.collisional_disk(600, seed=45, radius_scale=3000.0)
    want = oracle.direct_forces(d.px, d.py, d.pz, d.mass, d.active, 1e-4, radius=d.radius,
                                shell=True)
    for flag in (N.FLAG_ORDER_SIMD, N.FLAG_ORDER_PAIRWISE):
        got = _forces(engine, d, 1e-4, MODE_DIRECT_FP64 | FLAG_SHELL_THEOREM | flag)
        for g, w in zip(got, want):
            np.testing.assert_array_equal(g, w)


def test_known_answers(engine):
    """|a| = 1 for unit masses at distance 1 (test_gravity.cpp:16-45);
    inactive bodies get 0 (test_gravity.cpp:108-130); a lone body gets 0."""
    z2 = np.zeros(2)
    for mode in (MODE_DIRECT_FP64, MODE_DIRECT, MODE_BARNES_HUT, MODE_BARNES_HUT_REF):
        ax, ay, az = engine.compute_forces(np.array([-0.5, 0.5]), z2, z2, np.ones(2),
                                           np.ones(2, np.uint8), 0.0, mode)
        assert ax[0] == pytest.approx(1.0, rel=1e-6) and ax[1] == pytest.approx(-1.0, rel=1e-6)
        z3 = np.zeros(3)
        ax, ay, az = engine.compute_forces(np.array([0.0, 1.0, 2.0]), z3, z3, np.ones(3),
                                           np.array([1, 0, 1], np.uint8), 1e-4, mode)
        assert ax[1] == 0.0 and ay[1] == 0.0 and az[1] == 0.0
        ax, _, _ = engine.compute_forces(np.array([1.0]), np.zeros(1), np.zeros(1), np.ones(1),
                                         np.ones(1, np.uint8), 1e-4, mode)
        assert ax[0] == 0.0


@pytest.mark.parametrize("n", [1000, 50_000])
def test_direct_fp32_accuracy(engine, oracle, n):
    b = scenarios.plummer(n, seed=3)
    b.active[::97] = 0
    got = _forces(engine, b, 1e-4, MODE_DIRECT)
    if n <= 5000:
        want = oracle.direct_forces(b.px, b.py, b.pz, b.mass, b.active, 1e-4)
        e = rel_err(got, want)[b.active == 1]
    else:
        t = np.nonzero(b.active)[0][::37]
        want = oracle.direct_forces_targets(b.px, b.py, b.pz, b.mass, b.active, 1e-4, t)
        e = rel_err([g[t] for g in got], want)
    assert np.sqrt(np.mean(e ** 2)) < 2e-6
    assert e.max() < 1e-4


def test_direct_fp32_shell(engine, oracle):
    d = scenarios.collisional_disk(3000, seed=4, radius_scale=3000.0)
    got = _forces(engine, d, 1e-4, MODE_DIRECT | FLAG_SHELL_THEOREM)
    want = oracle.direct_forces(d.px, d.py, d.pz, d.mass, d.active, 1e-4, radius=d.radius,
                                shell=True)
    e = rel_err(got, want)
    assert np.sqrt(np.mean(e ** 2)) < 1e-5


def test_bh_reference_mode_matches_reference_solver(engine, ref_lib):
    b = scenarios.plummer(6000, seed=31)
    b.active[::41] = 0
    got = _forces(engine, b, 1e-4, MODE_BARNES_HUT_REF, theta=0.5)
    (want, _, _) = ref_lib.ref_bh_forces(b.px, b.py, b.pz, b.mass, b.active, 1e-4, 0.5)
    e = rel_err(got, want)[b.active == 1]
    assert e.max() < 1e-9


def test_bh_reference_mode_matches_oracle_golden(engine, oracle):
    from pathlib import Path

    g = dict(np.load(Path(__file__).parent / "golden" / "plummer512_bh.npz"))
    engine.set_param(N.PARAM_THETA, 0.5)
    got = engine.compute_forces(g["px"], g["py"], g["pz"], g["m"], g["active"], float(g["eps"]),
                                MODE_BARNES_HUT_REF)
    e = rel_err(got, [g["ax"], g["ay"], g["az"]])
    assert e.max() < 1e-9


def test_bh_reference_mode_shell(engine, oracle):
    d = scenarios.collisional_disk(2000, seed=6, radius_scale=3000.0)
    got = _forces(engine, d, 1e-4, MODE_BARNES_HUT_REF | FLAG_SHELL_THEOREM, theta=0.5)
    want = oracle.bh_forces(d.px, d.py, d.pz, d.mass, d.active, 1e-4, 0.5, radius=d.radius,
                            shell=True)
    e = rel_err(got, want)
    assert e.max() < 1e-9


@pytest.mark.parametrize("mode,tol", [(MODE_DIRECT, 1e-5), (MODE_BARNES_HUT, 1e-3)])
def test_zero_softening(engine, oracle, mode, tol):
    # eps = 0: the self pair must give 0 (not 0 * inf) in every packed path
    b = scenarios.plummer(5000, seed=9)
    got = _forces(engine, b, 0.0, mode)
    want = oracle.direct_forces(b.px, b.py, b.pz, b.mass, b.active, 0.0)
    assert all(np.all(np.isfinite(g)) for g in got)
    e = rel_err(got, want)
    assert np.sqrt(np.mean(e ** 2)) < tol


def test_group_work_bounded_at_2m(engine):
    # A walk group packed from sparse siblings must not enclose a dense
    # sibling: at N = 2^21 (seed 1) such a group once walked to every body.
    n = 1 << 21
    b = scenarios.plummer(n, seed=1)
    engine.set_param(N.PARAM_THETA, 0.5)
    engine.set_state(b, old_acc=False)
    engine.step(1, 0.0, 1e-4, MODE_BARNES_HUT)
    c = engine.counters()
    assert c[N.C_MAX_GROUP_WORK] < 20_000, c[N.C_MAX_GROUP_WORK]
    assert c[N.C_GROUPS] < n // 16  # packing still fills the warps


@pytest.mark.parametrize("n", [20_000, 200_000])
def test_bh_group_walk_error_budget(engine, oracle, n):
    b = scenarios.plummer(n, seed=1)
    t = np.arange(0, n, max(1, n // 2048))
    want = oracle.direct_forces_targets(b.px, b.py, b.pz, b.mass, b.active, 1e-4, t)
    errs = {}
    for quad in (True, False):
        flags = MODE_BARNES_HUT | (0 if quad else FLAG_NO_QUADRUPOLE)
        got = _forces(engine, b, 1e-4, flags, theta=0.5)
        errs[quad] = np.sqrt(np.mean(rel_err([g[t] for g in got], want) ** 2))
    assert errs[True] < 1e-3
    assert errs[True] < errs[False]
    c = engine.counters()
    assert c[N.C_CELL_INTERACTIONS] > 0 and c[N.C_BODY_INTERACTIONS] > 0


@pytest.mark.parametrize("n", [50_001, 200_000])
def test_bh_group_sizes_32_and_64(engine, oracle, n):
    """Walk groups of up to 32 bodies (one per lane) and of up to 64 (two per
    lane, the default): both within the theta = 0.5 error budget, each run to
    run bit-identical, and the larger group (a looser group box) never less
    accurate by more than a few percent."""
    b = scenarios.plummer(n, seed=6)
    t = np.arange(0, n, max(1, n // 2048))
    want = oracle.direct_forces_targets(b.px, b.py, b.pz, b.mass, b.active, 1e-4, t)
    errs = {}
    try:
        for gb in (32, 64):
            engine.set_param(N.PARAM_GROUP_BODIES, gb)
            got = _forces(engine, b, 1e-4, MODE_BARNES_HUT, theta=0.5)
            again = _forces(engine, b, 1e-4, MODE_BARNES_HUT, theta=0.5)
            for x, y in zip(got, again):
                np.testing.assert_array_equal(x, y)
            errs[gb] = np.sqrt(np.mean(rel_err([g[t] for g in got], want) ** 2))
            assert errs[gb] < 1e-3, (gb, errs[gb])
            groups = engine.counters()[N.C_GROUPS]
            assert groups >= -(-n // gb)
    finally:
        engine.set_param(N.PARAM_GROUP_BODIES, 64)
    assert errs[64] < errs[32] * 1.05


def test_bh_group_walk_theta_monotone(engine, oracle):
    b = scenarios.plummer(30_000, seed=2)
    t = np.arange(0, 30_000, 29)
    want = oracle.direct_forces_targets(b.px, b.py, b.pz, b.mass, b.active, 1e-4, t)
    prev = np.inf
    for th in (0.9, 0.7, 0.5, 0.3):
        got = _forces(engine, b, 1e-4, MODE_BARNES_HUT, theta=th)
        rms = np.sqrt(np.mean(rel_err([g[t] for g in got], want) ** 2))
        assert rms <= prev * 1.05
        prev = rms


def test_bh_group_walk_shell_and_inactive(engine, oracle):
    d = scenarios.collisional_disk(20_000, seed=8, radius_scale=1500.0)
    d.active[::11] = 0
    got = _forces(engine, d, 1e-4, MODE_BARNES_HUT | FLAG_SHELL_THEOREM, theta=0.5)
    t = np.nonzero(d.active)[0][::7]
    want = oracle.direct_forces_targets(d.px, d.py, d.pz, d.mass, d.active, 1e-4, t,
                                        radius=d.radius, shell=True)
    e = rel_err([g[t] for g in got], want)
    assert np.sqrt(np.mean(e ** 2)) < 1e-3
    assert np.all(got[0][d.active == 0] == 0.0)


def test_bh_deterministic_run_to_run(engine):
    b = scenarios.plummer(100_000, seed=5)
    a1 = _forces(engine, b, 1e-4, MODE_BARNES_HUT)
    a2 = _forces(engine, b, 1e-4, MODE_BARNES_HUT)
    for x, y in zip(a1, a2):
        np.testing.assert_array_equal(x, y)


def test_errors_reported(engine):
    b = scenarios.plummer(100, seed=1)
    b.px[3] = np.nan
    with pytest.raises(NBodyError) as e:
        _forces(engine, b, 1e-4, MODE_BARNES_HUT)
    assert e.value.status == N.NB_ERR_NONFINITE
    with pytest.raises(NBodyError) as e:
        big = np.zeros(engine.capacity + 1)
        engine.compute_forces(big, big, big, big, np.ones(len(big), np.uint8), 1e-4, MODE_DIRECT)
    assert e.value.status == N.NB_ERR_CAPACITY
    # the handle stays usable after an error
    b = scenarios.plummer(100, seed=1)
    _forces(engine, b, 1e-4, MODE_BARNES_HUT)
