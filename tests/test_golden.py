"""The oracle restatement against golden fixtures produced by the reference's
own CPU code (tests/golden/make_golden.py).  Runs without the reference."""
from __future__ import annotations

from pathlib import Path

import numpy as np

GOLD = Path(__file__).resolve().parent / "golden"


def _load(name):
    return dict(np.load(GOLD / name))


def test_trig_octree_and_forces(oracle):
    g = _load("trig200_bh.npz")
    t = oracle.octree(g["px"], g["py"], g["pz"], g["m"], g["active"])
    for k in ("center", "mass", "com", "children", "body", "leaf"):
        np.testing.assert_array_equal(t[k], g["t_" + k], err_msg=k)
    for th, sfx in ((0.5, "05"), (0.0, "00")):
        a = oracle.bh_forces(g["px"], g["py"], g["pz"], g["m"], g["active"], float(g["eps"]), th)
        for c, x in zip("xyz", a):
            np.testing.assert_array_equal(x, g[f"a{c}{sfx}"])


def test_plummer_octree_and_forces(oracle):
    g = _load("plummer512_bh.npz")
    t = oracle.octree(g["px"], g["py"], g["pz"], g["m"], g["active"])
    for k in ("center", "mass", "com", "children", "body", "leaf"):
        np.testing.assert_array_equal(t[k], g["t_" + k], err_msg=k)
    a = oracle.bh_forces(g["px"], g["py"], g["pz"], g["m"], g["active"], float(g["eps"]), 0.5)
    for c, x in zip("xyz", a):
        np.testing.assert_array_equal(x, g["a" + c])


def test_compaction(oracle):
    g = _load("compact3000.npz")
    dest, kept = oracle.compact_indices(g["in_active"], g["in_mass"])
    assert kept == int(g["kept"])
    sel = dest >= 0
    for k in ("px", "py", "pz", "vx", "vy", "vz", "mass"):
        out = np.empty(kept)
        out[dest[sel]] = g["in_" + k][sel]
        np.testing.assert_array_equal(out, g["out_" + k])


def test_merges(oracle):
    g = _load("merge_disk2000.npz")
    b = {k: g["in_" + k] for k in ("px", "py", "pz", "vx", "vy", "vz", "mass", "radius",
                                    "density", "active")}
    lo, hi = oracle.broad_phase(b["px"], b["py"], b["pz"], b["radius"], b["active"])
    np.testing.assert_array_equal(lo, g["lo"])
    np.testing.assert_array_equal(hi, g["hi"])
    out, k = oracle.resolve_merges(b, lo, hi)
    assert k == int(g["merges"])
    for key in out:
        np.testing.assert_array_equal(out[key], g["out_" + key], err_msg=key)
