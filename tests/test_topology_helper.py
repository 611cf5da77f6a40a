"""The vectorised topology comparison of tests/helpers.py (used at 1,048,576
bodies against the reference's own OctreeBuilder) checked on the CPU: the
engine's tree form (single-child chains collapsed, children contiguous,
bodies in key order) is built here from the oracle's pool octree; it must
compare equal, and a planted mistake must be found."""
from __future__ import annotations

import numpy as np

from helpers import topology_mismatches
from nbody_b200 import scenarios


def engine_form(pool, keys):
    """Walk-tree arrays of a pool octree (OctreeBuilder layout, one body per
    leaf): a node is kept where the cell splits or a body is alone, at the
    level of its deepest cell; children in Morton digit order."""
    ch, body, leaf = pool["children"], pool["body"], pool["leaf"].astype(bool)
    order = np.argsort(keys, kind="stable")
    rank = np.empty_like(order)
    rank[order] = np.arange(len(order))
    level, first, nch, bfirst, bcount = [], [], [], [], []
    morton_child = [0, 4, 2, 6, 1, 5, 3, 7]  # octant x+2y+4z -> digit 4x+2y+z order

    def bodies_of(k):
        if leaf[k]:
            return [int(body[k])]
        out = []
        for o in range(8):
            c = ch[k][o]
            if c >= 0:
                out += bodies_of(int(c))
        return out

    def emit(k, depth):
        # collapse single-child chains
        while not leaf[k]:
            kids = [int(c) for c in ch[k] if c >= 0]
            if len(kids) != 1:
                break
            k, depth = kids[0], depth + 1
        idx = len(level)
        bs = sorted(bodies_of(k), key=lambda b: rank[b])
        level.append(depth)
        first.append(-1)
        nch.append(0)
        bfirst.append(int(rank[bs[0]]))
        bcount.append(len(bs))
        if leaf[k]:
            return idx
        kids = []
        for d in range(8):
            o = morton_child.index(d)  # octant whose Morton digit is d
            c = ch[k][o]
            if c >= 0:
                kids.append(int(c))
        return idx, kids, depth

    # breadth-first over kept nodes so that children are contiguous
    out = emit(0, 0)
    queue = [out] if isinstance(out, tuple) else []
    while queue:
        idx, kids, depth = queue.pop(0)
        first[idx] = len(level)
        nch[idx] = len(kids)
        for c in kids:
            r = emit(c, depth + 1)
            if isinstance(r, tuple):
                queue.append(r)
    return {"level": np.array(level), "first_child": np.array(first),
            "n_children": np.array(nch), "body_first": np.array(bfirst),
            "body_count": np.array(bcount), "n_nodes": len(level),
            "sorted_idx": order.astype(np.int32), "sorted_keys": keys[order]}


def test_helper_equal_on_an_exact_copy_and_finds_a_planted_mistake(oracle):
    b = scenarios.plummer(3000, seed=41)
    pool = oracle.octree(b.px, b.py, b.pz, b.mass, b.active)
    keys, _, _ = oracle.morton_cube(b.px, b.py, b.pz, b.active)
    form = engine_form(pool, keys)
    mm = topology_mismatches(pool, form, b.px, b.py, b.pz)
    assert mm["cells"] == 0 and mm["bodies"] == 0, mm
    # planted: two bodies in different leaves trade places in the sorted order
    bad = dict(form)
    sidx = form["sorted_idx"].copy()
    sidx[[10, 2000]] = sidx[[2000, 10]]
    bad["sorted_idx"] = sidx
    mm = topology_mismatches(pool, bad, b.px, b.py, b.pz)
    assert mm["bodies"] >= 2
    # planted: one body's leaf one level too deep
    bad = dict(form)
    lv = form["level"].copy()
    leafs = np.nonzero(form["n_children"] == 0)[0]
    lv[leafs[5]] += 1
    bad["level"] = lv
    mm = topology_mismatches(pool, bad, b.px, b.py, b.pz)
    assert mm["cells"] > 0 and mm["bodies"] >= 1
