"""Batched ensembles on the GPU against the FP64 oracle, system by system.

Tolerances: direct systems (FP32 pair forces on FP64-differenced
coordinates, compensated tile sums) rms relative error <= 1e-5 and max
<= 1e-4 against the FP64 direct sum; tree systems (theta 0.5, monopole +
quadrupole) rms <= 1e-3; energies (FP64) to 1e-12 relative."""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from helpers import rel_err
from nbody_b200 import Ensemble, scenarios
from nbody_b200 import _native as N

pytestmark = pytest.mark.gpu
EPS = 1e-4


def _systems(sizes, seed=3, spread=0.0):
    out = []
    for s, k in enumerate(sizes):
        b = scenarios.plummer(int(k), 1.0, 1.0, seed=seed * 1000 + s)
        if spread:
            b.px += spread * s  # systems may overlap or sit apart: they never interact
        out.append(b)
    return out


def _per_system_errors(ens, systems, max_targets=512):
    st = ens.get_state()
    errs = []
    for s, b in enumerate(systems):
        o0, o1 = ens.offsets[s], ens.offsets[s + 1]
        t = np.unique(np.linspace(0, b.n - 1, min(b.n, max_targets)).astype(np.int64))
        want = oracle.direct_forces_targets(b.px, b.py, b.pz, b.mass, b.active, EPS, t)
        got = [st[k][o0:o1][t] for k in ("ax", "ay", "az")]
        e = rel_err(got, want)
        errs.append((np.sqrt(np.mean(e ** 2)), e.max()))
    return errs


def test_direct_systems_match_oracle():
    sizes = [64, 65, 127, 300, 1000, 2048]
    systems = _systems(sizes)
    with Ensemble(sizes, ds_max_n=2048) as ens:
        assert ens.info()["tree_systems"] == 0
        ens.set_state(systems)
        ens.compute_forces(EPS)
        for rms, mx in _per_system_errors(ens, systems):
            assert rms < 1e-5 and mx < 1e-4, (rms, mx)


def test_tree_systems_match_oracle():
    sizes = [2049, 3000, 5000, 8192]
    systems = _systems(sizes, seed=4)
    with Ensemble(sizes, ds_max_n=2048) as ens:
        assert ens.info()["tree_systems"] == 4
        ens.set_state(systems)
        ens.compute_forces(EPS)
        for rms, _ in _per_system_errors(ens, systems):
            assert rms < 1e-3, rms
        c = ens.counters()
        assert c["tree_cell"] > 0 and c["tree_body"] > 0


@pytest.mark.parametrize("spread", [0.0, 0.5, 40.0])
def test_mixed_systems_stay_isolated(spread):
    # interleaved direct and tree systems, overlapping in space (spread 0),
    # touching, or far apart: each sees only its own bodies
    sizes = [2500, 64, 4000, 700, 3000, 2048, 100]
    systems = _systems(sizes, seed=5, spread=spread)
    with Ensemble(sizes, ds_max_n=2048) as ens:
        ens.set_state(systems)
        ens.compute_forces(EPS)
        for s, (rms, mx) in enumerate(_per_system_errors(ens, systems)):
            bound = 1e-5 if sizes[s] <= 2048 else 1e-3
            assert rms < bound, (s, rms)
        # the engine's own FP64 audit agrees with the oracle-based check
        rms_dev, _ = ens.force_error(256, 7, EPS)
        assert np.all(rms_dev[np.array(sizes) <= 2048] < 1e-5)
        assert np.all(rms_dev[np.array(sizes) > 2048] < 1e-3)


def test_zero_softening():
    sizes = [300, 2500]
    systems = _systems(sizes, seed=9)
    with Ensemble(sizes, ds_max_n=2048) as ens:
        ens.set_state(systems)
        ens.compute_forces(0.0)
        st = ens.get_state()
        for s, b in enumerate(systems):
            o0, o1 = ens.offsets[s], ens.offsets[s + 1]
            want = oracle.direct_forces(b.px, b.py, b.pz, b.mass, b.active, 0.0)
            got = [st[k][o0:o1] for k in ("ax", "ay", "az")]
            assert all(np.all(np.isfinite(g)) for g in got)
            rms = np.sqrt(np.mean(rel_err(got, want) ** 2))
            assert rms < (1e-5 if sizes[s] <= 2048 else 1e-3), (s, rms)


def test_every_direct_shape_and_autotune():
    sizes = [64, 200, 513, 1024, 2000]
    systems = _systems(sizes, seed=6)
    with Ensemble(sizes, ds_max_n=2048) as ens:
        ens.set_state(systems)
        for shape in range(len(N.ENS_SHAPES)):
            ens.set_param(N.PARAM_ENS_DIRECT_SHAPE, shape)
            ens.compute_forces(EPS)
            assert ens.counters()["direct_shape"] == shape
            for rms, mx in _per_system_errors(ens, systems, 128):
                assert rms < 1e-5 and mx < 1e-4, (shape, rms, mx)
        best, ms = ens.autotune(EPS)
        assert 0 <= best < len(N.ENS_SHAPES) and ms[best] > 0
        assert ms[best] == ms[ms > 0].min()
        assert ens.counters()["direct_shape"] == best


def test_energy_matches_oracle_and_steps_conserve_it():
    sizes = [64, 900, 2048, 2600, 6000]
    systems = _systems(sizes, seed=7)
    with Ensemble(sizes, ds_max_n=2048) as ens:
        ens.set_state(systems)
        e0, ke0, pe0 = ens.energy(EPS)
        for s, b in enumerate(systems):
            d = {k: getattr(b, k) for k in ("px", "py", "pz", "vx", "vy", "vz", "mass", "active")}
            want = oracle.energy(d, EPS)
            assert ke0[s] == pytest.approx(want["ke"], rel=1e-12)
            assert pe0[s] == pytest.approx(want["pe"], rel=1e-12)
        ens.step(200, 1e-4, EPS)
        assert ens.counters()["graph_launches"] == 200
        assert ens.ms_per_step() > 0
        e1, _, _ = ens.energy(EPS)
        drift = np.abs((e1 - e0) / e0)
        assert np.all(drift < 1e-5), drift
        st = ens.get_state()
        assert np.all(np.isfinite(st["px"])) and np.all(np.isfinite(st["ax"]))


def test_step_is_velocity_verlet():
    # one step by hand from the ensemble's own forces: x1 = x0 + dt (v0 + dt/2 a0),
    # v1 = v0 + dt/2 (a0 + a1)
    sizes = [300, 2100]
    systems = _systems(sizes, seed=8)
    dt = 1e-3
    with Ensemble(sizes, ds_max_n=2048) as ens:
        ens.set_state(systems)
        ens.compute_forces(EPS)
        s0 = ens.get_state()
        ens.step(1, dt, EPS)
        s1 = ens.get_state()
        for k, v, a in (("px", "vx", "ax"), ("py", "vy", "ay"), ("pz", "vz", "az")):
            x1 = s0[k] + dt * (s0[v] + 0.5 * dt * s0[a])
            np.testing.assert_allclose(s1[k], x1, rtol=0, atol=1e-15 * (1 + np.abs(x1).max()))
            v1 = s0[v] + 0.5 * dt * (s0[a] + s1[a])
            np.testing.assert_allclose(s1[v], v1, rtol=1e-12, atol=1e-15)


def test_rejects_bad_input():
    from nbody_b200.engine import NBodyError
    with pytest.raises(NBodyError):
        Ensemble([64, 0, 10])
    with Ensemble([64, 100]) as ens:
        with pytest.raises(NBodyError):
            ens.step(1, 1e-3, EPS)  # no state yet
        b = _systems([64, 100])
        b[1].px[3] = np.nan
        with pytest.raises(NBodyError):
            ens.set_state(b)


def test_tree_autotune_choices_keep_systems_apart_and_accurate():
    """nb_ens_autotune_tree times every (walk block shape, walk-group span,
    group size) it may use on the current state and keeps the fastest.  A span at or
    above the smallest tree system's size is never tried (its groups could
    take bodies of two systems) and is refused as a parameter; every tried
    configuration gives each tree system its theta = 0.5 accuracy."""
    sizes = [100, 2049, 3000, 5000, 8192]
    systems = _systems(sizes, seed=6, spread=0.5)
    with Ensemble(sizes, ds_max_n=2048) as ens:
        ens.set_state(systems)
        choice, ms = ens.autotune_tree(EPS)
        assert 0 <= choice < len(N.ENS_TREE_CHOICES)
        assert ms[choice] > 0 and ms[choice] == min(m for m in ms if m > 0)
        # every span below 2049 is tried for both block shapes
        assert np.all(ms > 0)
        for k, (shape, span, bodies) in enumerate(N.ENS_TREE_CHOICES):
            ens.set_param(N.PARAM_ENS_WALK_SHAPE, shape)
            ens.set_param(N.PARAM_GROUP_SPAN, span)
            ens.set_param(N.PARAM_GROUP_BODIES, bodies)
            ens.compute_forces(EPS)
            errs = _per_system_errors(ens, systems)
            for s, (rms, mx) in enumerate(errs):
                bound = 1e-5 if sizes[s] <= 2048 else 1e-3
                assert rms < bound, (k, s, rms)
    with Ensemble([100, 300], ds_max_n=64) as small:
        # tree systems of 100 and 300 bodies: spans of 128 and up are refused
        with pytest.raises(Exception):
            small.set_param(N.PARAM_GROUP_SPAN, 128)
        small.set_param(N.PARAM_GROUP_SPAN, 64)
        small.set_state(_systems([100, 300], seed=7))
        choice, ms = small.autotune_tree(EPS)
        # only sibling packing (span 0) is tried, for both block shapes
        assert choice in (0, 4) and ms[0] > 0 and ms[4] > 0
        assert all(ms[k] == -1 for k in (1, 2, 3, 5, 6, 7, 8, 9, 10))
