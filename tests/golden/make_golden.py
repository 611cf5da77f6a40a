"""Generate the golden fixtures from the reference's own CPU code.

Runs oracle/_ref/libcelestial_ref.so (the reference engine's octree builder,
Barnes-Hut solver, compaction and merge resolver, compiled in place from the
reference sources) on small deterministic inputs and stores inputs and
outputs in tests/golden/*.npz.  The fixtures pin the oracle restatement
where the reference tree is not available (tests/test_golden.py).

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "oracle"))
sys.path.insert(0, str(ROOT / "celestial-mechanics-desktop_b200"))

import oracle  # noqa: E402
from nbody_b200 import scenarios  # noqa: E402

OUT = Path(__file__).resolve().parent


def trig_bodies(n: int):
    """Deterministic fixture of the reference's gravity / validation tests
    (engine/tests/test_gravity.cpp:67-75)."""
    i = np.arange(n, dtype=np.float64)
    return (np.sin(i * 1.0) * 10.0, np.cos(i * 1.3) * 10.0, np.sin(i * 0.7) * 10.0,
            1.0 + np.abs(np.sin(i * 2.0)))


def main():
    if oracle.ref() is None:
        raise SystemExit("oracle/_ref not built: run make -C oracle ref")
    # 1. trig fixture: octree + BH forces (theta 0.5 and 0.0 -> clamped 0.2)
    px, py, pz, m = trig_bodies(200)
    act = np.ones(200, np.uint8)
    act[7] = 0
    t = oracle.ref_octree(px, py, pz, m, act)
    (a05, _, _) = oracle.ref_bh_forces(px, py, pz, m, act, 1e-4, 0.5)
    (a00, _, _) = oracle.ref_bh_forces(px, py, pz, m, act, 1e-4, 0.0)
    np.savez_compressed(OUT / "trig200_bh.npz", px=px, py=py, pz=pz, m=m, active=act,
                        eps=1e-4, ax05=a05[0], ay05=a05[1], az05=a05[2], ax00=a00[0],
                        ay00=a00[1], az00=a00[2], t_center=t["center"], t_mass=t["mass"],
                        t_com=t["com"], t_children=t["children"], t_body=t["body"],
                        t_leaf=t["leaf"])
    # 2. Plummer N=512, seed 0: octree + BH forces
    b = scenarios.plummer(512, 1.0, 1.0, seed=0)
    t = oracle.ref_octree(b.px, b.py, b.pz, b.mass, b.active)
    (a, _, _) = oracle.ref_bh_forces(b.px, b.py, b.pz, b.mass, b.active, 1e-4, 0.5)
    np.savez_compressed(OUT / "plummer512_bh.npz", px=b.px, py=b.py, pz=b.pz, m=b.mass,
                        active=b.active, eps=1e-4, ax=a[0], ay=a[1], az=a[2],
                        t_center=t["center"], t_mass=t["mass"], t_com=t["com"],
                        t_children=t["children"], t_body=t["body"], t_leaf=t["leaf"])
    # 3. compaction: ParticleSystem::compact
    rng = np.random.Generator(np.random.PCG64(5))
    n = 3000
    arrs = {k: rng.standard_normal(n) for k in ("px", "py", "pz", "vx", "vy", "vz")}
    mass = rng.uniform(0.1, 1.0, n)
    act = (rng.random(n) > 0.3).astype(np.uint8)
    c = {k: v.copy() for k, v in arrs.items()}
    mc, ac = mass.copy(), act.copy()
    import ctypes as C  # noqa: F401
    p = lambda a: a.ctypes.data  # noqa: E731
    kept = oracle.ref().ref_compact(n, p(c["px"]), p(c["py"]), p(c["pz"]), p(c["vx"]),
                                    p(c["vy"]), p(c["vz"]), p(mc), p(ac))
    np.savez_compressed(OUT / "compact3000.npz", **{f"in_{k}": v for k, v in arrs.items()},
                        in_mass=mass, in_active=act, kept=kept,
                        **{f"out_{k}": v[:kept] for k, v in c.items()}, out_mass=mc[:kept],
                        out_active=ac[:kept])
    # 4. merges: CollisionResolver::resolve (Merge mode) on a dense cluster
    d = scenarios.collisional_disk(2000, seed=7, radius_scale=2000.0)
    lo, hi = oracle.broad_phase(d.px, d.py, d.pz, d.radius, d.active, d.collidable)
    bd = {k: getattr(d, k) for k in ("px", "py", "pz", "vx", "vy", "vz", "mass", "radius",
                                      "density", "active")}
    out, k = oracle.ref_resolve_merges(bd, lo, hi)
    np.savez_compressed(OUT / "merge_disk2000.npz", **{f"in_{k2}": v for k2, v in bd.items()},
                        lo=lo, hi=hi, merges=k, **{f"out_{k2}": v for k2, v in out.items()})
    print("pairs", len(lo), "merges", k)


if __name__ == "__main__":
    main()
