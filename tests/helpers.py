"""Canonical octree forms and small numeric helpers for the tests."""
from __future__ import annotations

import numpy as np


def compact21(v: np.ndarray) -> np.ndarray:
    """De-interleave every third bit (inverse of the Morton spread)."""
    v = v.astype(np.uint64) & np.uint64(0x1249249249249249)
    v = (v | (v >> np.uint64(2))) & np.uint64(0x10C30C30C30C30C3)
    v = (v | (v >> np.uint64(4))) & np.uint64(0x100F00F00F00F00F)
    v = (v | (v >> np.uint64(8))) & np.uint64(0x1F0000FF0000FF)
    v = (v | (v >> np.uint64(16))) & np.uint64(0x1F00000000FFFF)
    v = (v | (v >> np.uint64(32))) & np.uint64(0x1FFFFF)
    return v


def ref_canonical(tree: dict, max_depth: int = 21) -> set:
    """{(depth, ix, iy, iz, bodies)} of a reference pool octree
    (OctreeBuilder::build layout: node 0 is the root, children[8], body)."""
    c4, ch, body, leaf = tree["center"], tree["children"], tree["body"], tree["leaf"]
    root = c4[0]
    lo = root[:3] - root[3]
    out = set()

    def walk(k, depth):
        bodies = []
        if leaf[k]:
            bodies = [int(body[k])]
        else:
            for c in ch[k]:
                if c >= 0:
                    bodies += walk(int(c), depth + 1)
        if depth <= max_depth:
            w = 2.0 * root[3] / (1 << depth)
            idx = tuple(int(np.rint((c4[k][a] - lo[a]) / w - 0.5)) for a in range(3))
            out.add((depth, *idx, tuple(sorted(bodies))))
        return bodies

    import sys
    old = sys.getrecursionlimit()
    sys.setrecursionlimit(max(old, 10000))
    try:
        walk(0, 0)
    finally:
        sys.setrecursionlimit(old)
    return out


def gpu_canonical(t: dict) -> set:
    """Same canonical form from the engine's walk tree (built with leaf
    capacity 1): single-child chains are expanded back level by level."""
    level, fc, nc = t["level"], t["first_child"], t["n_children"]
    bf, bc = t["body_first"], t["body_count"]
    sidx, skeys = t["sorted_idx"], t["sorted_keys"]
    kx = compact21(skeys >> np.uint64(2))
    ky = compact21(skeys >> np.uint64(1))
    kz = compact21(skeys)
    parent_level = np.full(t["n_nodes"], -1, np.int64)
    for k in range(t["n_nodes"]):
        if nc[k] > 0:
            parent_level[fc[k]:fc[k] + nc[k]] = level[k]
    out = set()
    for k in range(t["n_nodes"]):
        bodies = tuple(sorted(int(x) for x in sidx[bf[k]:bf[k] + bc[k]]))
        b0 = bf[k]
        for d in range(parent_level[k] + 1, level[k] + 1):
            s = np.uint64(21 - d)
            out.add((d, int(kx[b0] >> s), int(ky[b0] >> s), int(kz[b0] >> s), bodies))
    return out


def rel_err(a, b):
    """Per-body |a-b|/|b| for stacked (3, n) arrays."""
    a = np.asarray(a)
    b = np.asarray(b)
    num = np.sqrt(((a - b) ** 2).sum(axis=0))
    den = np.sqrt((b ** 2).sum(axis=0))
    return num / np.where(den > 0, den, 1.0)


def trig_bodies(n: int):
    """Deterministic fixture of engine/tests/test_gravity.cpp:67-75."""
    i = np.arange(n, dtype=np.float64)
    return (np.sin(i * 1.0) * 10.0, np.cos(i * 1.3) * 10.0, np.sin(i * 0.7) * 10.0,
            1.0 + np.abs(np.sin(i * 2.0)))
