"""The decision rule of the parallel merge (k_merge_rounds in
celestial-mechanics-desktop_b200/csrc/collide.cu), restated here in Python,
against the oracle's sequential CollisionResolver restatement (which is
pinned to the reference's own resolver): on random conflict-heavy pair
lists, with windows smaller than the pair list and binding per-frame and
per-body caps, the rounds merge exactly the pairs the sequential loop
merges, with the same survivors.  CPU only; the GPU kernel itself is checked
against the oracle in tests/test_gpu_step.py."""
from __future__ import annotations

import numpy as np
import pytest


def merge_rounds(n, pairs, mass, active, max_frame, max_body, window):
    """Windows of `window` pairs; per round a pending pair is ready when it is
    the lowest pending pair touching each of its bodies; with E merges among
    resolved earlier pairs and U earlier pending pairs, it decides when
    E >= max_frame (skip) or E + U < max_frame, else waits."""
    m, act = mass.copy(), active.copy()
    cnt = np.zeros(n, np.int64)
    merged, base, npairs = 0, 0, len(pairs)
    while base < npairs and merged < max_frame:
        ks = range(base, min(base + window, npairs))
        pending = {k: True for k in ks}
        event = {k: False for k in ks}
        for _ in range(window + 1):
            if not any(pending.values()):
                break
            owner = {}
            for k in ks:
                if pending[k]:
                    for x in pairs[k]:
                        owner[x] = min(owner.get(x, 1 << 60), k)
            pend_before, ev_before, pc, ec = {}, {}, 0, 0
            for k in ks:
                pend_before[k], ev_before[k] = pc, ec
                pc += pending[k]
                ec += event[k]
            decided = []
            for k in ks:
                a, b = pairs[k]
                if not pending[k] or owner[a] != k or owner[b] != k:
                    continue
                e = merged + ev_before[k]
                if not act[a] or not act[b] or e >= max_frame:
                    decided.append((k, False))
                elif e + pend_before[k] < max_frame:
                    decided.append((k, cnt[a] < max_body and cnt[b] < max_body))
            for k, do in decided:
                pending[k] = False
                if not do:
                    continue
                a, b = pairs[k]
                total = m[a] + m[b]
                if not total < 1e-30:
                    sv, vc = (a, b) if m[a] >= m[b] else (b, a)
                    m[sv] = total
                    act[vc] = 0
                cnt[a if (m[a] > 0 and act[a]) else b] += 1
                event[k] = True
        else:
            raise AssertionError("a round resolved no pair")
        merged += sum(event.values())
        base += window
    return m, act, merged


@pytest.mark.parametrize("seed", range(12))
def test_rounds_equal_the_sequential_resolver(oracle, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    n = int(rng.integers(8, 80))
    want_pairs = int(rng.integers(10, 500))
    pr = set()
    while len(pr) < min(want_pairs, n * (n - 1) // 2):
        a, b = sorted(rng.choice(n, 2, replace=False).tolist())
        pr.add((a, b))
    pairs = sorted(pr)
    mass = (rng.choice([0.0, 1.0, 2.0, 3.0], n) if seed % 3 == 0 else rng.random(n) + 0.1)
    active = (rng.random(n) > 0.1).astype(np.uint8)
    max_frame = int(rng.choice([1, 3, 10, 64]))
    max_body = int(rng.choice([1, 2, 3]))
    window = int(rng.choice([4, 16, 1024]))
    b = {"px": rng.random(n), "py": rng.random(n), "pz": rng.random(n), "vx": rng.random(n),
         "vy": rng.random(n), "vz": rng.random(n), "mass": mass, "radius": rng.random(n) * 0.1,
         "density": np.zeros(n), "active": active}
    lo = np.array([p[0] for p in pairs], np.int32)
    hi = np.array([p[1] for p in pairs], np.int32)
    out, nm = oracle.resolve_merges(b, lo, hi, max_frame=max_frame, max_body=max_body)
    m, act, merged = merge_rounds(n, pairs, mass.copy(), active.copy(), max_frame, max_body,
                                  window)
    assert merged == nm
    np.testing.assert_array_equal(act, out["active"])
    np.testing.assert_array_equal(m, out["mass"])
