"""ctypes loader of the oracle libraries.  TEST INFRASTRUCTURE ONLY.

liboracle.so        - C restatement of the reference arithmetic (nbody_oracle.c)
_ref/libcelestial_ref.so - the reference's own CPU code compiled in place
                      (ref_harness.cpp); optional (absent when the reference
                      tree was not available at build time).
Only tests, the smoke check and the benchmark's CPU-baseline leg use this.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
REF_LIB = HERE / "_ref" / "libcelestial_ref.so"
REF_GPU_LIB = HERE / "_ref" / "libcelestial_ref_gpu.so"
# root of the reference repository (only needed to build _ref)
REF_ENV = "CELESTIAL_REF"

P = C.c_void_p
i32, f64, u8 = C.c_int32, C.c_double, C.c_uint8


def build(ref: bool = True) -> None:
    """Compile liboracle.so, and _ref when $CELESTIAL_REF names the
    reference repository root and its engine sources are there."""
    root = os.environ.get(REF_ENV, "")
    with_ref = ref and root and (Path(root) / "engine" / "src").is_dir()
    targets = ["all"] + (["ref", f"CELESTIAL_REF={root}"] if with_ref else [])
    subprocess.run(["make", "-s", "-C", str(HERE), *targets], check=True)


def _p(a):
    return None if a is None else a.ctypes.data


def _load(path: Path, sigs: dict):
    lib = C.CDLL(str(path))
    for name, (res, args) in sigs.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


_OR_SIGS = {
    "or_direct_forces": (None, [i32, P, P, P, P, P, P, f64, i32, P, P, P, i32]),
    "or_direct_forces_targets": (None, [i32, P, P, P, P, P, P, f64, i32, i32, P, P, P, P, i32]),
    "or_bbox": (None, [i32, P, P, P, P, P]),
    "or_cube_from_bbox": (None, [P, P]),
    "or_morton_aabb": (None, [i32, P, P, P, P, P, P, P]),
    "or_morton_cube": (None, [i32, P, P, P, P, P, P, P]),
    "or_stable_sort": (None, [i32, P, P]),
    "or_octree_build": (i32, [i32, P, P, P, P, P, f64, i32, P, P, P, P, P, P]),
    "or_bh_forces": (None, [i32, P, P, P, P, P, f64, f64, i32, P, P, P, P, P, P, P, P, P, i32]),
    "or_compact_indices": (i32, [i32, P, P, P]),
    "or_broad_phase": (i32, [i32, P, P, P, P, P, P, i32, P, P]),
    "or_resolve_merges": (i32, [i32, P, P, P, P, P, P, P, P, P, P, i32, P, P, i32, i32, i32, f64]),
    "or_verlet_direct": (None, [i32, P, P, P, P, P, P, P, P, P, P, P, f64, f64, i32, i32]),
    "or_energy": (None, [i32, P, P, P, P, P, P, P, P, f64, P, i32]),
    "or_yoshida_direct": (None, [i32, P, P, P, P, P, P, P, P, P, P, P, f64, f64, i32, i32]),
    "or_adaptive_dt": (f64, [i32, P, P, P, P, f64, f64, f64, f64]),
    "or_force_error": (i32, [i32, P, P, P, P, P, P, P, P]),
    "or_direct_forces_order": (None, [i32, P, P, P, P, P, P, f64, i32, i32, P, P, P, i32]),
    "or_verlet_direct_order": (None, [i32, P, P, P, P, P, P, P, P, P, P, P, f64, f64, i32, i32,
                                      i32]),
    "or_yoshida_direct_order": (None, [i32, P, P, P, P, P, P, P, P, P, P, P, f64, f64, i32, i32,
                                       i32]),
    "or_energy_tracker": (None, [i32, P, P, P, P, P, P, P, P, f64, P]),
    "or_broad_phase_parallel": (i32, [i32, P, P, P, P, P, P, i32, P, P, i32]),
}
_REF_SIGS = {
    "ref_morton_from_unit": (C.c_uint64, [f64, f64, f64]),
    "ref_octree_build": (i32, [i32, P, P, P, P, P, f64, i32, P, P, P, P, P, P]),
    "ref_bh_forces": (f64, [i32, P, P, P, P, P, f64, f64, i32, i32, P, P, P, P]),
    "ref_compact": (i32, [i32, P, P, P, P, P, P, P, P]),
    "ref_resolve_merges": (i32, [i32, P, P, P, P, P, P, P, P, P, P, i32, P, P, i32, i32, i32, f64]),
    "ref_engine_steps": (i32, [i32, P, P, P, P, P, P, P, P, P, P, P, P, i32, i32, f64, f64, f64,
                               i32]),
    "ref_engine_update": (i32, [i32, P, P, P, P, P, P, P, P, P, P, P, i32, i32, f64, f64, f64,
                                i32, f64, f64, f64, f64, f64, i32, P, P]),
    "ref_energy_tracker": (None, [i32, P, P, P, P, P, P, P, P, f64, P]),
}

_REF_GPU_SIGS = {
    "ref_gpu_gravity": (i32, [i32, P, P, P, P, P, f64, i32, P, P, P, P]),
    "ref_gpu_radix_sort": (i32, [i32, P, P, P]),
    "ref_gpu_tree": (i32, [i32, P, P, P, P, P, f64, f64, i32, P, P, P, P, P, P]),
}

_lib = None
_ref = None
_ref_gpu = None


def lib():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build(ref=False)
        _lib = _load(LIB, _OR_SIGS)
    return _lib


def ref():
    """The reference's own CPU code, or None when it was not built."""
    global _ref
    if _ref is None and REF_LIB.exists():
        _ref = _load(REF_LIB, _REF_SIGS)
    return _ref


def ref_gpu():
    """Two of the reference's own CUDA kernels (FP64 gravity, radix sort)
    built for sm_100a, or None when they were not built.  Loading it needs a
    CUDA runtime; calling it needs a GPU."""
    global _ref_gpu
    if _ref_gpu is None and REF_GPU_LIB.exists():
        _ref_gpu = _load(REF_GPU_LIB, _REF_GPU_SIGS)
    return _ref_gpu


def ref_gpu_gravity(px, py, pz, m, active, eps, reps=3):
    """The reference's tiled FP64 gravity kernel on the current GPU: the
    accelerations and the mean time per launch (ms)."""
    n = len(px)
    px, py, pz, m = map(_f, (px, py, pz, m))
    act = _u8(active)
    ax, ay, az = np.empty(n), np.empty(n), np.empty(n)
    ms = np.zeros(1)
    r = ref_gpu().ref_gpu_gravity(n, _p(px), _p(py), _p(pz), _p(m), _p(act), eps, int(reps),
                                  _p(ax), _p(ay), _p(az), _p(ms))
    if r != 0:
        raise RuntimeError("reference gravity kernel failed")
    return (ax, ay, az), float(ms[0])


def ref_gpu_tree(px, py, pz, m, active, eps, theta=0.5, reps=1):
    """The reference's GpuTreeSolver::compute_forces on the current GPU (one
    untimed evaluation, then `reps` timed ones): the accelerations, the mean
    time per evaluation (ms, CUDA events) and the solver's own
    sort+build / traversal split of the last one (ms, host clock)."""
    n = len(px)
    px, py, pz, m = map(_f, (px, py, pz, m))
    act = _u8(active)
    ax, ay, az = np.empty(n), np.empty(n), np.empty(n)
    ms, build, trav = np.zeros(1), np.zeros(1), np.zeros(1)
    r = ref_gpu().ref_gpu_tree(n, _p(px), _p(py), _p(pz), _p(m), _p(act), eps, theta, int(reps),
                               _p(ax), _p(ay), _p(az), _p(ms), _p(build), _p(trav))
    if r != 0:
        raise RuntimeError("reference GPU tree solver failed")
    return (ax, ay, az), float(ms[0]), float(build[0]), float(trav[0])


def ref_gpu_radix_sort(keys, values):
    """The reference's launch_radix_sort on the current GPU: its output
    (keys, values) and the time (ms)."""
    k = np.ascontiguousarray(keys, np.uint64).copy()
    v = np.ascontiguousarray(values, np.int32).copy()
    ms = np.zeros(1)
    if ref_gpu().ref_gpu_radix_sort(len(k), _p(k), _p(v), _p(ms)) != 0:
        raise RuntimeError("reference radix sort failed")
    return k, v, float(ms[0])


def _f(a, n=None):
    return np.ascontiguousarray(a, np.float64)


def _u8(a):
    return np.ascontiguousarray(a, np.uint8)


def threads() -> int:
    return os.cpu_count() or 1


# ---- wrappers -------------------------------------------------------------

def direct_forces(px, py, pz, m, active, eps, radius=None, shell=False, nthreads=None):
    n = len(px)
    px, py, pz, m = map(_f, (px, py, pz, m))
    active = _u8(active)
    radius = None if radius is None else _f(radius)
    ax, ay, az = np.empty(n), np.empty(n), np.empty(n)
    lib().or_direct_forces(n, _p(px), _p(py), _p(pz), _p(m), _p(radius), _p(active), eps,
                           int(shell), _p(ax), _p(ay), _p(az), nthreads or threads())
    return ax, ay, az


def direct_forces_targets(px, py, pz, m, active, eps, targets, radius=None, shell=False,
                          nthreads=None):
    n = len(px)
    px, py, pz, m = map(_f, (px, py, pz, m))
    active = _u8(active)
    t = np.ascontiguousarray(targets, np.int32)
    ax, ay, az = np.empty(len(t)), np.empty(len(t)), np.empty(len(t))
    radius = None if radius is None else _f(radius)
    lib().or_direct_forces_targets(n, _p(px), _p(py), _p(pz), _p(m), _p(radius), _p(active),
                                   eps, int(shell), len(t), _p(t), _p(ax), _p(ay), _p(az),
                                   nthreads or threads())
    return ax, ay, az


def bbox(px, py, pz, active):
    out = np.empty(6)
    px, py, pz = map(_f, (px, py, pz))
    lib().or_bbox(len(px), _p(px), _p(py), _p(pz), _p(_u8(active)), _p(out))
    return out


def cube_from_bbox(b):
    out = np.empty(4)
    lib().or_cube_from_bbox(_p(_f(b)), _p(out))
    return out


def morton_aabb(px, py, pz, active):
    n = len(px)
    b = bbox(px, py, pz, active)
    keys = np.empty(n, np.uint64)
    idx = np.empty(n, np.int32)
    px, py, pz = map(_f, (px, py, pz))
    lib().or_morton_aabb(n, _p(px), _p(py), _p(pz), _p(_u8(active)), _p(b), _p(keys), _p(idx))
    return keys, idx


def morton_cube(px, py, pz, active, cube=None):
    n = len(px)
    if cube is None:
        cube = cube_from_bbox(bbox(px, py, pz, active))
    cube = _f(cube)
    keys = np.empty(n, np.uint64)
    idx = np.empty(n, np.int32)
    px, py, pz = map(_f, (px, py, pz))
    lib().or_morton_cube(n, _p(px), _p(py), _p(pz), _p(_u8(active)), _p(cube), _p(keys), _p(idx))
    return keys, idx, cube


def stable_sort(keys, values):
    k = np.ascontiguousarray(keys, np.uint64).copy()
    v = np.ascontiguousarray(values, np.int32).copy()
    lib().or_stable_sort(len(k), _p(k), _p(v))
    return k, v


def _octree(fn, px, py, pz, m, active, min_node_size=1e-12, cap=None):
    n = len(px)
    cap = cap or (4 * n + 64)
    c4 = np.empty((cap, 4))
    mass = np.empty(cap)
    com = np.empty((cap, 3))
    ch = np.empty((cap, 8), np.int32)
    body = np.empty(cap, np.int32)
    leaf = np.empty(cap, np.uint8)
    px, py, pz, m = map(_f, (px, py, pz, m))
    k = fn(n, _p(px), _p(py), _p(pz), _p(m), _p(_u8(active)), min_node_size, cap, _p(c4),
           _p(mass), _p(com), _p(ch), _p(body), _p(leaf))
    if k < 0:
        raise RuntimeError("octree pool too small")
    return dict(center=c4[:k], mass=mass[:k], com=com[:k], children=ch[:k], body=body[:k],
                leaf=leaf[:k])


def octree(px, py, pz, m, active, min_node_size=1e-12):
    return _octree(lib().or_octree_build, px, py, pz, m, active, min_node_size)


def ref_octree(px, py, pz, m, active, min_node_size=1e-12):
    return _octree(ref().ref_octree_build, px, py, pz, m, active, min_node_size)


def bh_forces(px, py, pz, m, active, eps, theta, radius=None, shell=False, tree=None,
              nthreads=None):
    n = len(px)
    t = tree or octree(px, py, pz, m, active)
    px, py, pz = map(_f, (px, py, pz))
    radius = None if radius is None else _f(radius)
    ax, ay, az = np.empty(n), np.empty(n), np.empty(n)
    c4 = np.ascontiguousarray(t["center"])
    com = np.ascontiguousarray(t["com"])
    ch = np.ascontiguousarray(t["children"])
    lib().or_bh_forces(n, _p(px), _p(py), _p(pz), _p(radius), _p(_u8(active)), eps, theta,
                       int(shell), _p(c4), _p(t["mass"]), _p(com), _p(ch), _p(t["body"]),
                       _p(t["leaf"]), _p(ax), _p(ay), _p(az), nthreads or threads())
    return ax, ay, az


def ref_bh_forces(px, py, pz, m, active, eps, theta, parallel=False, nthreads=0):
    n = len(px)
    px, py, pz, m = map(_f, (px, py, pz, m))
    ax, ay, az = np.empty(n), np.empty(n), np.empty(n)
    bms = np.zeros(1)
    trav = ref().ref_bh_forces(n, _p(px), _p(py), _p(pz), _p(m), _p(_u8(active)), eps, theta,
                               int(parallel), int(nthreads), _p(ax), _p(ay), _p(az), _p(bms))
    return (ax, ay, az), float(bms[0]), float(trav)


def compact_indices(active, mass):
    dest = np.empty(len(active), np.int32)
    k = lib().or_compact_indices(len(active), _p(_u8(active)), _p(_f(mass)), _p(dest))
    return dest, int(k)


def broad_phase(px, py, pz, radius, active, collidable=None, max_pairs=1 << 22,
                nthreads=None):
    """All pairs with |xi - xj|^2 < (ri + rj)^2 in (lo, hi) order; the rows
    are split over `nthreads` threads when given (same list)."""
    lo = np.empty(max_pairs, np.int32)
    hi = np.empty(max_pairs, np.int32)
    px, py, pz, radius = map(_f, (px, py, pz, radius))
    act = _u8(active)
    col = None if collidable is None else _u8(collidable)
    if nthreads:
        k = lib().or_broad_phase_parallel(len(px), _p(px), _p(py), _p(pz), _p(radius), _p(act),
                                          _p(col), max_pairs, _p(lo), _p(hi), int(nthreads))
    else:
        k = lib().or_broad_phase(len(px), _p(px), _p(py), _p(pz), _p(radius), _p(act),
                                 _p(col), max_pairs, _p(lo), _p(hi))
    k = min(k, max_pairs)
    return lo[:k].copy(), hi[:k].copy()


def _merge(fn, b: dict, lo, hi, max_frame=64, max_body=2, density_merge=1, min_radius=1e-6):
    arrs = {k: _f(b[k]).copy() for k in ("px", "py", "pz", "vx", "vy", "vz", "mass", "radius",
                                          "density")}
    act = _u8(b["active"]).copy()
    lo = np.ascontiguousarray(lo, np.int32)
    hi = np.ascontiguousarray(hi, np.int32)
    k = fn(len(act), *(_p(arrs[k]) for k in ("px", "py", "pz", "vx", "vy", "vz", "mass",
                                              "radius", "density")), _p(act), len(lo), _p(lo),
           _p(hi), max_frame, max_body, density_merge, min_radius)
    arrs["active"] = act
    return arrs, int(k)


def resolve_merges(b, lo, hi, **kw):
    return _merge(lib().or_resolve_merges, b, lo, hi, **kw)


def ref_resolve_merges(b, lo, hi, **kw):
    return _merge(ref().ref_resolve_merges, b, lo, hi, **kw)


# direct-sum orders of the reference backends (or_direct_forces_order)
ORDER_PARALLEL, ORDER_SIMD, ORDER_PAIRWISE = 0, 1, 2
_STATE = ("px", "py", "pz", "vx", "vy", "vz", "ax", "ay", "az", "mass")


def direct_forces_order(px, py, pz, m, active, eps, order, radius=None, shell=False,
                        nthreads=None):
    """Direct sum in the order of CpuParallelBackend (0), the SIMD backend /
    native engine (1) or CpuSingleThreadBackend (2)."""
    n = len(px)
    px, py, pz, m = map(_f, (px, py, pz, m))
    active = _u8(active)
    radius = None if radius is None else _f(radius)
    ax, ay, az = np.empty(n), np.empty(n), np.empty(n)
    lib().or_direct_forces_order(n, _p(px), _p(py), _p(pz), _p(m), _p(radius), _p(active), eps,
                                 int(shell), int(order), _p(ax), _p(ay), _p(az),
                                 nthreads or threads())
    return ax, ay, az


def verlet_direct(b: dict, eps, dt, steps, nthreads=None, order=ORDER_PARALLEL):
    a = {k: _f(b[k]).copy() for k in _STATE}
    act = _u8(b["active"])
    lib().or_verlet_direct_order(len(act), *(_p(a[k]) for k in _STATE), _p(act), eps, dt, steps,
                                 int(order), nthreads or threads())
    return a


def yoshida_direct(b: dict, eps, dt, steps, nthreads=None, order=ORDER_PARALLEL):
    a = {k: _f(b[k]).copy() for k in _STATE}
    act = _u8(b["active"])
    lib().or_yoshida_direct_order(len(act), *(_p(a[k]) for k in _STATE), _p(act), eps, dt, steps,
                                  int(order), nthreads or threads())
    return a


def ref_engine_steps(b: dict, eps, dt, steps, compute_mode=0, integrator=0, theta=0.5):
    """The reference's own Engine (CPU_BruteForce = 0 / CPU_BarnesHut = 1,
    Leapfrog_KDK = 0 / Yoshida4 = 1): set_particles, then `steps` steps."""
    a = {k: _f(b[k]).copy() for k in _STATE}
    act = _u8(b["active"])
    rad = _f(b["radius"]) if b.get("radius") is not None else None
    r = ref().ref_engine_steps(len(act), *(_p(a[k]) for k in _STATE), _p(rad), _p(act),
                               int(compute_mode), int(integrator), theta, dt, eps, int(steps))
    if r != 0:
        raise RuntimeError("reference Engine threw")
    return a


def ref_engine_update(b: dict, eps, dt, frame_time, frames, compute_mode=0, integrator=0,
                      theta=0.5, adaptive=False, eta=0.01, dt_min=1e-8, dt_max=0.01,
                      initial_dt=0.001):
    """`frames` calls of the reference Engine::update(frame_time); returns
    (final state, steps per frame, adaptive dt after the last frame)."""
    a = {k: _f(b[k]).copy() for k in _STATE}
    act = _u8(b["active"])
    steps = np.zeros(frames, np.int32)
    dt_out = np.zeros(1)
    r = ref().ref_engine_update(len(act), *(_p(a[k]) for k in _STATE), _p(act),
                                int(compute_mode), int(integrator), theta, dt, eps,
                                int(adaptive), eta, dt_min, dt_max, initial_dt, frame_time,
                                int(frames), _p(steps), _p(dt_out))
    if r != 0:
        raise RuntimeError("reference Engine threw")
    return a, steps, float(dt_out[0])


_ENERGY_KEYS = ("ke", "pe", "e", "px", "py", "pz", "lx", "ly", "lz", "comx", "comy", "comz", "m")


def _energy_args(b):
    # hold the converted arrays: ctypes gets raw pointers
    arrs = [_f(b[k]) for k in ("px", "py", "pz", "vx", "vy", "vz", "mass")]
    return arrs, _u8(b["active"])


def energy_tracker(b: dict, eps):
    """The native engine's EnergyTracker::compute restated (or_energy_tracker)."""
    out = np.empty(13)
    arrs, act = _energy_args(b)
    lib().or_energy_tracker(len(act), *(_p(x) for x in arrs), _p(act), eps, _p(out))
    return dict(zip(_ENERGY_KEYS, out.tolist()))


def ref_energy_tracker(b: dict, eps):
    """EnergyTracker::compute of the reference itself."""
    out = np.empty(13)
    arrs, act = _energy_args(b)
    ref().ref_energy_tracker(len(act), *(_p(x) for x in arrs), _p(act), eps, _p(out))
    return dict(zip(_ENERGY_KEYS, out.tolist()))


def adaptive_dt(b: dict, eps, eta, dt_min, dt_max):
    ax, ay, az = (_f(b[k]) for k in ("ax", "ay", "az"))
    act = _u8(b["active"])  # held: the library reads it during the call
    return lib().or_adaptive_dt(len(ax), _p(ax), _p(ay), _p(az), _p(act), eps, eta, dt_min,
                                dt_max)


def energy(b: dict, eps, nthreads=None):
    out = np.empty(13)
    arrs, act = _energy_args(b)
    lib().or_energy(len(act), *(_p(x) for x in arrs), _p(act), eps, _p(out),
                    nthreads or threads())
    return dict(zip(_ENERGY_KEYS, out.tolist()))


def force_error(a, ref_a, active=None):
    out = np.empty(3)
    ax, ay, az = map(_f, a)
    rx, ry, rz = map(_f, ref_a)
    act = None if active is None else _u8(active)
    lib().or_force_error(len(ax), _p(ax), _p(ay), _p(az), _p(rx), _p(ry), _p(rz), _p(act),
                         _p(out))
    return tuple(out.tolist())
