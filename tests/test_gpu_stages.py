"""Integer stages on the GPU against the oracle: Morton keys, stable sort,
octree topology, compaction indices, broad-phase pairs.  Bit-exact."""
from __future__ import annotations

import numpy as np
import pytest

from helpers import gpu_canonical, ref_canonical, trig_bodies
from nbody_b200 import scenarios

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [1, 2, 255, 4097, 100_003])
def test_morton_aabb_bit_exact(engine, oracle, n):
    b = scenarios.plummer(n, seed=n)
    if n > 3:
        b.active[1::9] = 0
    keys, idx, _ = engine.morton_keys(b.px, b.py, b.pz, b.active, 0)
    want, widx = oracle.morton_aabb(b.px, b.py, b.pz, b.active)
    np.testing.assert_array_equal(keys, want)
    np.testing.assert_array_equal(idx, widx)


@pytest.mark.parametrize("n", [3, 5000, 262_145])
def test_morton_cube_bit_exact(engine, oracle, n):
    b = scenarios.plummer(n, seed=7 + n)
    b.active[::13] = 0
    keys, _, cube = engine.morton_keys(b.px, b.py, b.pz, b.active, 1)
    want, _, wcube = oracle.morton_cube(b.px, b.py, b.pz, b.active)
    np.testing.assert_array_equal(cube, wcube)
    np.testing.assert_array_equal(keys, want)


def test_morton_degenerate_box(engine, oracle):
    """All bodies on one point (range 0 -> inverse range 0, morton_kernel.cu:61-63)."""
    n = 100
    px = np.full(n, 3.0)
    z = np.zeros(n)
    act = np.ones(n, np.uint8)
    keys, _, _ = engine.morton_keys(px, z, z, act, 0)
    want, _ = oracle.morton_aabb(px, z, z, act)
    np.testing.assert_array_equal(keys, want)


@pytest.mark.parametrize("n,dup", [(0, 0), (1, 0), (2, 1), (4095, 0), (4097, 1), (300_001, 1),
                                   (400_003, 0), (1_000_003, 1), (2_000_000, 0)])
def test_stable_sort_bit_exact(engine, oracle, n, dup):
    """Tiles of 1024 keys (4097, 300,001), 2048 (400,003) and 4096 (1,000,003,
    2M) on a 148-SM B200; duplicates and sentinel keys keep their input order."""
    rng = np.random.Generator(np.random.PCG64(n))
    if dup:
        keys = rng.integers(0, 300, n).astype(np.uint64) * np.uint64(0x0123456789AB)
    else:
        keys = rng.integers(0, 2 ** 63, n, dtype=np.uint64)
    if n > 10:
        keys[:5] = np.uint64(0xFFFFFFFFFFFFFFFF)  # inactive sentinel keys
    vals = np.arange(n, dtype=np.int32)
    k, v = engine.sort_pairs(keys, vals)
    wk, wv = oracle.stable_sort(keys, vals)
    np.testing.assert_array_equal(k, wk)
    np.testing.assert_array_equal(v, wv)


def _topology_case(engine, oracle, px, py, pz, m, act):
    cube = oracle.cube_from_bbox(oracle.bbox(px, py, pz, act))
    t = engine.build_octree(px, py, pz, m, act, leaf_capacity=1, cube=cube)
    ref = oracle.octree(px, py, pz, m, act)
    got = gpu_canonical(t)
    want = ref_canonical(ref)
    assert got == want
    return t, ref


def test_octree_topology_trig(engine, oracle):
    px, py, pz, m = trig_bodies(300)
    act = np.ones(300, np.uint8)
    act[11] = 0
    _topology_case(engine, oracle, px, py, pz, m, act)


@pytest.mark.parametrize("n,seed", [(2, 1), (3, 2), (1000, 3), (20_000, 4)])
def test_octree_topology_plummer(engine, oracle, n, seed):
    b = scenarios.plummer(n, seed=seed)
    t, ref = _topology_case(engine, oracle, b.px, b.py, b.pz, b.mass, b.active)
    # root mass / centre of mass (OctreeBuilder::update_mass) to FP64 rounding
    assert t["mass"][0] == pytest.approx(ref["mass"][0], rel=1e-13)
    np.testing.assert_allclose(t["com"][0], ref["com"][0], rtol=0, atol=1e-12)


def test_octree_topology_reference_code(engine, ref_lib):
    """Against the reference's own OctreeBuilder (oracle/_ref)."""
    b = scenarios.plummer(5000, seed=21)
    b.active[3::7] = 0
    cube = ref_lib.cube_from_bbox(ref_lib.bbox(b.px, b.py, b.pz, b.active))
    t = engine.build_octree(b.px, b.py, b.pz, b.mass, b.active, leaf_capacity=1, cube=cube)
    assert gpu_canonical(t) == ref_canonical(ref_lib.ref_octree(b.px, b.py, b.pz, b.mass, b.active))


@pytest.mark.parametrize("n,seed,inactive", [(5000, 21, 7), (1_048_576, 1, 0)])
def test_octree_topology_reference_code_at_scale(engine, ref_lib, n, seed, inactive):
    """The walk tree (leaf capacity 1) against the reference's own
    OctreeBuilder (oracle/_ref) up to the Barnes-Hut workload's size: the
    Plummer sphere of 1,048,576 bodies, seed 1.  Compared at depths <= 21
    (keys of 21 bits per axis): every (depth, cell, body count) node and
    every body's leaf cell.  Mismatch classes: bodies a few ulp from a cell
    plane, and everything else; both must be empty."""
    from helpers import topology_mismatches

    b = scenarios.plummer(n, 1.0, 1.0, seed=seed)
    if inactive:
        b.active[3::inactive] = 0
    cube = ref_lib.cube_from_bbox(ref_lib.bbox(b.px, b.py, b.pz, b.active))
    t = engine.build_octree(b.px, b.py, b.pz, b.mass, b.active, leaf_capacity=1, cube=cube)
    ref = ref_lib.ref_octree(b.px, b.py, b.pz, b.mass, b.active)
    mm = topology_mismatches(ref, t, b.px, b.py, b.pz)
    assert mm["cells"] == 0 and mm["bodies"] == 0, mm
    if n <= 5000:  # the vectorised form agrees with the set-of-bodies form
        assert gpu_canonical(t) == ref_canonical(ref)


def test_octree_single_body_and_duplicates(engine, oracle):
    t = engine.build_octree(np.array([1.0]), np.array([2.0]), np.array([3.0]), np.array([10.0]),
                            np.ones(1, np.uint8), leaf_capacity=8)
    assert t["n_nodes"] == 1 and t["body_count"][0] == 1 and t["mass"][0] == 10.0
    np.testing.assert_array_equal(t["com"][0], [1.0, 2.0, 3.0])
    # 40 coincident bodies plus spread ones: one level-21 bucket holds the 40
    b = scenarios.plummer(200, seed=5)
    b.px[:40] = 0.25
    b.py[:40] = -0.5
    b.pz[:40] = 0.125
    t = engine.build_octree(b.px, b.py, b.pz, b.mass, b.active, leaf_capacity=4)
    leaf = t["n_children"] == 0
    assert t["body_count"][leaf].sum() == 200
    big = leaf & (t["body_count"] > 4)
    assert np.all(t["level"][big] == 21) and t["body_count"][big].max() >= 40


@pytest.mark.parametrize("cap", [1, 8, 16])
def test_walk_tree_invariants_and_multipoles(engine, cap):
    b = scenarios.plummer(30_000, seed=9)
    t = engine.build_octree(b.px, b.py, b.pz, b.mass, b.active, leaf_capacity=cap)
    nn = t["n_nodes"]
    fc, nc, bf, bc = t["first_child"], t["n_children"], t["body_first"], t["body_count"]
    leaf = nc == 0
    assert np.all((bc[leaf] <= cap) | (t["level"][leaf] == 21))
    assert bc[leaf].sum() == 30_000
    # children contiguous, cover the parent's body range in order
    for k in np.nonzero(~leaf)[0][:2000]:
        ch = np.arange(fc[k], fc[k] + nc[k])
        assert bf[ch[0]] == bf[k] and bf[ch[-1]] + bc[ch[-1]] == bf[k] + bc[k]
        assert np.all(bf[ch[1:]] == bf[ch[:-1]] + bc[ch[:-1]])
        assert np.all(t["level"][ch] > t["level"][k])
    # mass / COM / traceless quadrupole of sampled nodes from their bodies
    sidx = t["sorted_idx"]
    rng = np.random.Generator(np.random.PCG64(0))
    for k in rng.choice(nn, 300, replace=False):
        rows = sidx[bf[k]:bf[k] + bc[k]]
        m = b.mass[rows]
        x = np.stack([b.px[rows], b.py[rows], b.pz[rows]], 1)
        M = m.sum()
        com = (m[:, None] * x).sum(0) / M
        assert t["mass"][k] == pytest.approx(M, rel=1e-12)
        np.testing.assert_allclose(t["com"][k], com, rtol=0, atol=1e-12 * max(1, np.abs(com).max()))
        d = x - com
        r2 = (d * d).sum(1)
        q = np.einsum("i,ij,ik->jk", m, 3 * d, d) - np.eye(3) * (m * r2).sum()
        want = np.array([q[0, 0], q[1, 1], q[2, 2], q[0, 1], q[0, 2], q[1, 2]])
        scale = (m * r2).sum() + 1e-300
        np.testing.assert_allclose(t["quad"][k], want, rtol=0, atol=2e-5 * scale + 1e-30)


@pytest.mark.parametrize("n", [0, 1, 4096, 4097, 300_001])
def test_compaction_indices_bit_exact(engine, oracle, n):
    rng = np.random.Generator(np.random.PCG64(n + 3))
    act = (rng.random(n) > 0.2).astype(np.uint8)
    mass = rng.uniform(0, 1, n)
    mass[::50] = 0.0  # active with zero mass: removed (compact_kernel.cu:39)
    dest, kept = engine.compact_indices(act, mass)
    wd, wk = oracle.compact_indices(act, mass)
    assert kept == wk
    np.testing.assert_array_equal(dest, wd)


@pytest.mark.parametrize("n,scale,seed", [(3000, 2500.0, 1), (20_000, 1500.0, 2)])
def test_broad_phase_all_pairs(engine, oracle, n, scale, seed):
    d = scenarios.collisional_disk(n, seed=seed, radius_scale=scale)
    d.active[5::31] = 0
    d.collidable[7::29] = 0
    lo, hi = engine.broad_phase(d.px, d.py, d.pz, d.radius, d.active, d.collidable)
    wlo, whi = oracle.broad_phase(d.px, d.py, d.pz, d.radius, d.active, d.collidable)
    assert len(wlo) > 10
    np.testing.assert_array_equal(lo, wlo)
    np.testing.assert_array_equal(hi, whi)


def test_broad_phase_capacity_error(engine):
    from nbody_b200 import NBodyError

    d = scenarios.collisional_disk(3000, seed=1, radius_scale=2500.0)
    with pytest.raises(NBodyError) as e:
        engine.broad_phase(d.px, d.py, d.pz, d.radius, d.active, max_pairs=5)
    assert e.value.status == -2
