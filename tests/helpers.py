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


def _ref_depth_cells(tree: dict):
    c4 = tree["center"]
    root = c4[0]
    lo = root[:3] - root[3]
    depth = np.rint(np.log2(root[3] / c4[:, 3])).astype(np.int64)
    w = 2.0 * root[3] / np.exp2(depth.astype(np.float64))
    cell = np.rint((c4[:, :3] - lo) / w[:, None] - 0.5).astype(np.int64)
    return depth, cell


def topology_mismatches(ref_tree: dict, gpu_tree: dict, px, py, pz, max_depth: int = 21) -> dict:
    """Vectorised comparison of the reference pool octree (OctreeBuilder,
    one body per leaf) with the engine's walk tree built with leaf capacity
    1, at depths <= max_depth (the engine's keys have 21 bits per axis, so
    deeper reference splits appear as level-21 buckets).  Returns the
    mismatch counts: `cells` (multiset of (depth, cell, body count) entries
    found in only one tree), `bodies` (bodies whose leaf cell, capped at
    max_depth, differs) and, of those, `on_cell_plane` (bodies within a few
    ulp of a cell plane at the first depth where the two trees disagree)."""
    # ---- reference: depth, cell, body count of every node ------------------
    depth, cell = _ref_depth_cells(ref_tree)
    ch, body, leaf = ref_tree["children"], ref_tree["body"], ref_tree["leaf"].astype(bool)
    nn = len(depth)
    count = np.where(leaf & (body >= 0), 1, 0).astype(np.int64)
    for d in range(int(depth.max()), -1, -1):
        idx = np.nonzero((depth == d) & ~leaf)[0]
        if len(idx) == 0:
            continue
        c = ch[idx]
        count[idx] = np.where(c >= 0, count[np.maximum(c, 0)], 0).sum(axis=1)
    keep = depth <= max_depth
    ref_rows = np.concatenate([depth[keep, None], cell[keep], count[keep, None]], axis=1)
    # per body: its leaf cell, capped at max_depth
    lk = np.nonzero(leaf & (body >= 0))[0]
    n = len(px)
    rb_depth = np.full(n, -1, np.int64)
    rb_cell = np.zeros((n, 3), np.int64)
    d = depth[lk]
    sh = np.maximum(d - max_depth, 0)
    rb_depth[body[lk]] = np.minimum(d, max_depth)
    rb_cell[body[lk]] = cell[lk] >> sh[:, None]
    # ---- engine: expand single-child chains level by level ---------------------
    level = gpu_tree["level"].astype(np.int64)
    fc, nc = gpu_tree["first_child"], gpu_tree["n_children"]
    bf, bc = gpu_tree["body_first"], gpu_tree["body_count"]
    sidx, skeys = gpu_tree["sorted_idx"], gpu_tree["sorted_keys"]
    k = gpu_tree["n_nodes"]
    parent_level = np.full(k, -1, np.int64)
    internal = np.nonzero(nc > 0)[0]
    child_of = np.repeat(internal, nc[internal])
    child_idx = _expand_ranges(fc[internal], nc[internal])
    parent_level[child_idx] = level[child_of]
    span = level - parent_level
    node_rep = np.repeat(np.arange(k), span)
    dep = _expand_ranges(parent_level + 1, span)
    key0 = skeys[bf[node_rep]]
    s = (np.uint64(21) - dep.astype(np.uint64))
    gx = (compact21(key0 >> np.uint64(2)) >> s).astype(np.int64)
    gy = (compact21(key0 >> np.uint64(1)) >> s).astype(np.int64)
    gz = (compact21(key0) >> s).astype(np.int64)
    gpu_rows = np.stack([dep, gx, gy, gz, bc[node_rep].astype(np.int64)], axis=1)
    # per body: the engine leaf's cell
    gl = np.nonzero(nc == 0)[0]
    gb_depth = np.full(n, -1, np.int64)
    gb_cell = np.zeros((n, 3), np.int64)
    rep = np.repeat(gl, bc[gl])
    pos = _expand_ranges(bf[gl].astype(np.int64), bc[gl].astype(np.int64))
    bodies = sidx[pos]
    lv = level[rep]
    key = skeys[pos]
    s2 = (np.uint64(21) - lv.astype(np.uint64))
    gb_depth[bodies] = lv
    gb_cell[bodies, 0] = (compact21(key >> np.uint64(2)) >> s2).astype(np.int64)
    gb_cell[bodies, 1] = (compact21(key >> np.uint64(1)) >> s2).astype(np.int64)
    gb_cell[bodies, 2] = (compact21(key) >> s2).astype(np.int64)
    # ---- compare ---------------------------------------------------------------
    a = np.unique(ref_rows, axis=0, return_counts=True)
    b = np.unique(gpu_rows, axis=0, return_counts=True)
    ra = {tuple(r): c for r, c in zip(a[0].tolist(), a[1].tolist())}
    rb = {tuple(r): c for r, c in zip(b[0].tolist(), b[1].tolist())}
    cells = sum(abs(ra.get(t, 0) - rb.get(t, 0)) for t in set(ra) | set(rb))
    active = rb_depth >= 0
    bad = np.nonzero(active & ((rb_depth != gb_depth) | np.any(rb_cell != gb_cell, axis=1)))[0]
    # a body within a few ulp of a cell plane at the shallowest depth where
    # its two leaf paths differ
    root = ref_tree["center"][0]
    lo = root[:3] - root[3]
    on_plane = 0
    p = np.stack([px, py, pz], axis=1)
    for i in bad:
        dmin = int(min(rb_depth[i], gb_depth[i]))
        for dd in range(1, dmin + 1):
            w = 2.0 * root[3] / (1 << dd)
            u = (p[i] - lo) / w
            if np.any(np.abs(u - np.rint(u)) < 1e-9 * np.maximum(1.0, np.abs(u))):
                on_plane += 1
                break
    return {"cells": int(cells), "bodies": int(len(bad)), "on_cell_plane": int(on_plane),
            "ref_nodes": int(nn), "gpu_nodes": int(k)}


def _expand_ranges(starts: np.ndarray, lens: np.ndarray) -> np.ndarray:
    """Concatenation of arange(s, s + l) for each (s, l), vectorised."""
    lens = np.asarray(lens, np.int64)
    starts = np.asarray(starts, np.int64)
    tot = int(lens.sum())
    if tot == 0:
        return np.zeros(0, np.int64)
    off = np.repeat(np.cumsum(lens) - lens, lens)
    return np.repeat(starts, lens) + (np.arange(tot) - off)
