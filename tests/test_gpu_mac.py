"""Learned MAC on the GPU: the tensor-core training kernel's gradient and the
walk's inference routine against the CPU oracle, and the harvest -> train ->
learned-walk pipeline.

Tolerances: gradients agree with the oracle (same BF16 rounding points,
float64 sums) to 2e-3 relative in norm per parameter block: what is left is
FP32 against float64 accumulation and the rare element whose FP32 value sits
on a BF16 rounding boundary and rounds the other way (one BF16 ulp, 2^-8,
of that element); predictions to 2e-2 in normalised units (FP32
accumulation order only)."""
from __future__ import annotations

import numpy as np
import pytest

import mac_oracle as M
from helpers import rel_err
from nbody_b200 import FLAG_LEARNED_MAC, MODE_BARNES_HUT, Engine, scenarios
from nbody_b200 import _native as N

pytestmark = pytest.mark.gpu


def _random_model(seed=5):
    rng = np.random.Generator(np.random.PCG64(seed))
    p = M.init_params(seed)
    norm = np.concatenate([rng.normal(0, 1, 8), rng.uniform(0.5, 2, 8), [-20.0, 4.0]]).astype(np.float32)
    X = (rng.normal(0, 1.5, (777, 8)) * norm[8:16] + norm[:8]).astype(np.float32)
    Y = rng.normal(-20, 4, 777).astype(np.float32)
    return p, norm, X, Y


def test_training_gradient_matches_oracle(engine):
    p, norm, X, Y = _random_model()
    engine.mac_set_params(np.concatenate([p, norm]))
    g, loss = engine.mac_gradient(X, Y)
    wl, wg, _ = M.forward_backward(p, norm, X, Y, bf=True)
    assert loss == pytest.approx(wl, rel=1e-4)
    errs = []
    for lo, hi in ((M.W1, M.B1), (M.B1, M.W2), (M.W2, M.B2), (M.B2, M.W3), (M.W3, M.B3),
                   (M.B3, M.NPARAM)):
        errs.append(np.linalg.norm(g[lo:hi] - wg[lo:hi]) / max(np.linalg.norm(wg[lo:hi]), 1e-30))
    assert max(errs) < 2e-3, errs


def test_training_is_bitwise_reproducible():
    """The gradient sums per-warp and per-block partials in a fixed order (no
    floating-point atomics): repeated gradients over many blocks' rows, and
    two trainings of the same harvested set from the same seed, agree bit
    for bit."""
    rng = np.random.Generator(np.random.PCG64(9))
    p, norm, _, _ = _random_model(8)
    X = (rng.normal(0, 1.5, (300_000, 8)) * norm[8:16] + norm[:8]).astype(np.float32)
    Y = rng.normal(-20, 4, 300_000).astype(np.float32)
    b = scenarios.plummer(20_000, seed=4)
    params = []
    for _ in range(2):
        with Engine(20_000) as e:
            e.mac_set_params(np.concatenate([p, norm]))
            g1, l1 = e.mac_gradient(X, Y)
            g2, l2 = e.mac_gradient(X, Y)
            np.testing.assert_array_equal(g1, g2)
            assert l1 == l2
            e.mac_clear()
            e.set_state(b, old_acc=False)
            e.step(1, 0.0, 1e-4, MODE_BARNES_HUT)
            assert e.mac_harvest(400_000, 0.5, 1, 1e-4) > 4096
            e.mac_train(2, 2048, 2e-3, seed=11)
            params.append((e.mac_get_params(), e.mac_get_screen()))
    np.testing.assert_array_equal(params[0][0], params[1][0])
    np.testing.assert_array_equal(params[0][1], params[1][1])


def test_inference_matches_oracle(engine):
    p, norm, X, Y = _random_model(6)
    engine.mac_set_params(np.concatenate([p, norm]))
    y = engine.mac_predict(X)
    _, _, wy = M.forward_backward(p, norm, X, Y, bf=True)
    assert np.max(np.abs(y - wy)) / norm[17] < 2e-2


def test_params_round_trip(engine):
    p, norm, _, _ = _random_model(7)
    engine.mac_set_params(np.concatenate([p, norm]))
    np.testing.assert_array_equal(engine.mac_get_params(), np.concatenate([p, norm]))


def test_screen_controls_network_calls():
    """The linear screen decides the band alone at margin 0 and never at
    margin +inf (the state nb_mac_set_params leaves); one-body cells never
    reach the network."""
    n = 20_000
    b = scenarios.plummer(n, seed=22)
    p, norm, _, _ = _random_model(8)
    with Engine(n) as e:
        e.mac_set_params(np.concatenate([p, norm]))
        assert np.isinf(e.mac_get_screen()[-1])
        e.set_state(b, old_acc=False)

        def evals():
            # dt = 0: the geometric step restores the same |a| estimate each time
            e.step(1, 0.0, 1e-4, MODE_BARNES_HUT)
            e.step(1, 0.0, 1e-4, MODE_BARNES_HUT | FLAG_LEARNED_MAC)
            return int(e.counters()[N.C_MAC_EVALS])

        all_rows = evals()
        assert all_rows > 0
        scr = np.array([0.1, 0.2, 0.3, 0, 0, 0, 0, 0, 0.5, 0.0], np.float32)
        e.mac_set_screen(scr)
        np.testing.assert_array_equal(e.mac_get_screen(), scr)
        assert evals() == 0
        scr[-1] = 1e3
        e.mac_set_screen(scr)
        assert evals() == all_rows


def test_audit_falls_back_to_geometric():
    """Every NB_PARAM_MAC_AUDIT_INTERVAL steps the learned MAC's forces are
    checked against the FP64 direct sum on sampled bodies; an audit over
    NB_PARAM_MAC_AUDIT_RMS switches the handle to the geometric MAC."""
    n = 20_000
    b = scenarios.plummer(n, seed=23)
    p, norm, _, _ = _random_model(9)
    learned = MODE_BARNES_HUT | FLAG_LEARNED_MAC
    with Engine(n) as e:
        e.mac_set_params(np.concatenate([p, norm]))
        e.set_state(b, old_acc=False)
        e.step(1, 0.0, 1e-4, MODE_BARNES_HUT)  # |a| estimate
        e.set_param(N.PARAM_MAC_AUDIT_INTERVAL, 2)
        e.set_param(N.PARAM_MAC_AUDIT_RMS, 1e6)
        e.step(4, 1e-5, 1e-4, learned)
        st = e.mac_audit_state()
        assert st["audits"] == 2 and not st["fallback"] and st["rms"] > 0.0
        assert e.counters()[N.C_MAC_EVALS] > 0
        # an unreachable bound: the first audit falls back, later steps are geometric
        e.set_param(N.PARAM_MAC_AUDIT_INTERVAL, 2)
        e.set_param(N.PARAM_MAC_AUDIT_RMS, 1e-12)
        e.step(2, 1e-5, 1e-4, learned)
        st = e.mac_audit_state()
        assert st["audits"] == 1 and st["fallback"]
        e.step(1, 1e-5, 1e-4, learned)
        c = e.counters()
        assert c[N.C_MAC_EVALS] == 0 and c[N.C_MAC_FALLBACK] == 1
        # a new interval clears the fallback
        e.set_param(N.PARAM_MAC_AUDIT_INTERVAL, 0)
        assert not e.mac_audit_state()["fallback"]
        e.step(1, 1e-5, 1e-4, learned)
        assert e.counters()[N.C_MAC_EVALS] > 0


@pytest.mark.parametrize("samples", [1, 700, 5000])
def test_audit_sums_match_fp64_force_error(samples):
    """The in-run audit sums its sample on the force evaluation's sorted copy
    (FP32 pair terms on tile-differenced FP64 coordinates, FP64 accumulation);
    its rms and max relative errors equal nb_force_error's FP64 direct-sum
    figures for the same sample to 1e-4 relative (the audit reference is within
    ~1e-6 of the FP64 sum, the errors measured are ~1e-3)."""
    n = 30_000
    b = scenarios.hernquist(n, seed=24)
    p, norm, _, _ = _random_model(11)
    learned = MODE_BARNES_HUT | FLAG_LEARNED_MAC
    with Engine(n) as e:
        e.mac_set_params(np.concatenate([p, norm]))
        e.set_param(N.PARAM_MAC_BUDGET, -3.0)
        e.set_state(b, old_acc=False)
        e.step(1, 0.0, 1e-4, MODE_BARNES_HUT)
        e.set_param(N.PARAM_MAC_AUDIT_INTERVAL, 3)
        e.set_param(N.PARAM_MAC_AUDIT_SAMPLES, samples)
        e.set_param(N.PARAM_MAC_AUDIT_RMS, 1e6)
        e.step(3, 1e-5, 1e-4, learned)
        st = e.mac_audit_state()
        assert st["audits"] == 1
        mean, mx, rms = e.force_error(samples, 0x5EED, 1e-4)
        assert rms > 0.0
        assert st["rms"] == pytest.approx(rms, rel=1e-4)
        assert st["max"] == pytest.approx(mx, rel=1e-4)


def test_harvest_train_and_learned_walk():
    """Harvest -> train -> learned walk on a 60K Plummer sphere; the trained
    criterion reaches the geometric walk's error at theta 0.7 (about the
    1e-3 operating point) with fewer interactions (what the network gains)."""
    import oracle
    n = 60_000
    b = scenarios.plummer(n, seed=21)
    with Engine(n) as e:
        e.set_param(N.PARAM_THETA, 0.5)
        e.set_state(b, old_acc=False)
        e.step(1, 0.0, 1e-4, MODE_BARNES_HUT)  # an acceleration estimate for the features
        got = e.mac_harvest(2_000_000, 0.5, 1, 1e-4)
        X, Y = e.mac_dataset()
        assert got > 10_000 and len(Y) == got
        # band: log2(2h/d) in [log2 0.35, log2 1.0)
        assert X[:, 0].min() >= np.log2(0.35) - 1e-3 and X[:, 0].max() < 1e-3
        # single-body cells are exact up to FP64 rounding of the centre of
        # mass (target at most ~2^-45 of |a|); for the others the error grows
        # with the cell's pull relative to the group's |a| and with its size
        # over its distance
        multi = X[:, 4] > 0.5
        assert np.all(Y[~multi] < -45)
        assert np.corrcoef(X[multi, 2], Y[multi])[0, 1] > 0.8
        assert np.corrcoef(X[multi, 0], Y[multi])[0, 1] > 0.2
        losses = e.mac_train(8, 2048, 2e-3, seed=3)
        assert losses[-1] < 0.8 * losses[0] and losses[-1] < 0.1
        screen = e.mac_get_screen()
        assert np.all(np.isfinite(screen)) and 0.0 < screen[-1] < 2.0

        t = np.arange(0, n, 37)
        want = oracle.direct_forces_targets(b.px, b.py, b.pz, b.mass, b.active, 1e-4, t)

        def run(flags):
            e.set_state(b, old_acc=False)
            e.step(1, 0.0, 1e-4, MODE_BARNES_HUT)
            e.step(1, 0.0, 1e-4, flags)
            st, _ = e.get_state()
            rms = np.sqrt(np.mean(rel_err([st.ax[t], st.ay[t], st.az[t]], want) ** 2))
            c = e.counters()
            return rms, int(c[N.C_CELL_INTERACTIONS] + c[N.C_BODY_INTERACTIONS]), int(c[N.C_MAC_EVALS])

        e.set_param(N.PARAM_THETA, 0.7)
        rms_g, inter_g, _ = run(MODE_BARNES_HUT)
        for budget in np.arange(-2.7, -4.51, -0.15):
            e.set_param(N.PARAM_MAC_BUDGET, budget)
            rms_l, inter_l, evals = run(MODE_BARNES_HUT | FLAG_LEARNED_MAC)
            if rms_l <= rms_g:
                break
        assert rms_l <= rms_g, (rms_l, rms_g)
        assert evals > 0
        assert inter_l < 0.85 * inter_g, (budget, inter_l, inter_g)
