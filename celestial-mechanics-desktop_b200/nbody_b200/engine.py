"""Python host layer over the C ABI.

`Engine` is a thin owner of one handle.  `B200PhysicsBackend` and
`B200SoAIntegrator` mirror the reference's force-backend seam
(src/CelestialMechanics.Physics/Solvers/IPhysicsComputeBackend.cs:21-34,
IGravityModelAwareBackend.cs:6-9) and integrator interface
(Integrators/ISoAIntegrator.cs), with the same names in snake case, the
same argument meaning and the same error behaviour: failures raise.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N
from .scenarios import Bodies


class NBodyError(RuntimeError):
    """A negative status from the engine; `.status` holds it."""

    def __init__(self, status: int, message: str):
        super().__init__(f"nbody_b200 status {status}: {message}")
        self.status = status


class Engine:
    """One engine handle: a CUDA stream and device buffers for `capacity` bodies."""

    def __init__(self, capacity: int, device: int = 0):
        h = C.c_void_p()
        st = N.lib.nb_create(int(capacity), int(device), C.byref(h))
        if st != N.NB_OK:
            raise NBodyError(st, "nb_create failed (no sm_100 device, or out of memory)")
        self._h = h
        self.capacity = int(capacity)

    # -- lifetime ---------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            N.lib.nb_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st: int):
        if st != N.NB_OK:
            msg = N.lib.nb_last_error(self._h)
            raise NBodyError(st, msg.decode() if msg else "")
        return st

    # -- parameters -------------------------------------------------------
    def set_param(self, param: int, value):
        if isinstance(value, float):
            self._check(N.lib.nb_set_param_f64(self._h, param, value))
        else:
            self._check(N.lib.nb_set_param_i32(self._h, param, int(value)))

    @property
    def stream(self) -> int:
        return N.lib.nb_stream(self._h) or 0

    def timings(self) -> np.ndarray:
        out = np.zeros(N.T_COUNT)
        self._check(N.lib.nb_get_timings(self._h, N.ptr(out), N.T_COUNT))
        return out

    def counters(self) -> np.ndarray:
        out = np.zeros(N.C_COUNT, np.int64)
        self._check(N.lib.nb_get_counters(self._h, N.ptr(out), N.C_COUNT))
        return out

    def adaptive_dt(self) -> float:
        """dt of the next FLAG_ADAPTIVE_DT step (0 before the first)."""
        out = np.zeros(1)
        self._check(N.lib.nb_get_adaptive_dt(self._h, N.ptr(out)))
        return float(out[0])

    # -- the seam -----------------------------------------------------------
    def compute_forces(self, px, py, pz, mass, active, softening: float, flags: int,
                       radius=None, out=None):
        n = len(px)
        px, py, pz, mass = (N.f64a(a, n) for a in (px, py, pz, mass))
        active = N.u8a(active, n)
        radius = None if radius is None else N.f64a(radius, n)
        ax, ay, az = out if out is not None else (np.empty(n), np.empty(n), np.empty(n))
        self._check(N.lib.nb_compute_forces(self._h, n, N.ptr(px), N.ptr(py), N.ptr(pz),
                                            N.ptr(mass), N.ptr(radius), N.ptr(active),
                                            float(softening), int(flags), N.ptr(ax), N.ptr(ay),
                                            N.ptr(az)))
        return ax, ay, az

    # -- device-resident state --------------------------------------------
    def set_state(self, b: Bodies, old_acc: bool = True):
        n = b.n
        arrs = [N.f64a(getattr(b, k), n) for k in ("px", "py", "pz", "vx", "vy", "vz", "mass")]
        rad = N.f64a(b.radius, n)
        dens = None if b.density is None else N.f64a(b.density, n)
        act = N.u8a(b.active, n)
        col = None if b.collidable is None else N.u8a(b.collidable, n)
        acc = [N.f64a(getattr(b, k), n) for k in ("ax", "ay", "az")] if old_acc else [None] * 3
        self._check(N.lib.nb_set_state(self._h, n, *(N.ptr(a) for a in arrs[:6]), N.ptr(arrs[6]),
                                       N.ptr(rad), N.ptr(dens), N.ptr(act), N.ptr(col),
                                       *(N.ptr(a) for a in acc)))

    def get_state(self) -> tuple[Bodies, np.ndarray]:
        n_out = np.zeros(1, np.int32)
        cap = self.capacity
        f = {k: np.empty(cap) for k in ("px", "py", "pz", "vx", "vy", "vz", "ax", "ay", "az",
                                         "mass", "radius")}
        act = np.empty(cap, np.uint8)
        ids = np.empty(cap, np.int32)
        self._check(N.lib.nb_get_state(self._h, N.ptr(n_out), *(N.ptr(f[k]) for k in (
            "px", "py", "pz", "vx", "vy", "vz", "ax", "ay", "az", "mass", "radius")),
            N.ptr(act), N.ptr(ids)))
        n = int(n_out[0])
        b = Bodies(**{k: v[:n].copy() for k, v in f.items()}, active=act[:n].copy())
        return b, ids[:n].copy()

    def step(self, n_steps: int, dt: float, softening: float, flags: int):
        self._check(N.lib.nb_step(self._h, int(n_steps), float(dt), float(softening), int(flags)))

    def diagnostics(self, softening: float, pe_mode: int = 0) -> dict:
        out = np.zeros(13)
        self._check(N.lib.nb_diagnostics(self._h, float(softening), int(pe_mode), N.ptr(out)))
        keys = ("ke", "pe", "e", "px", "py", "pz", "lx", "ly", "lz", "comx", "comy", "comz", "m")
        return dict(zip(keys, out.tolist()))

    def force_error(self, n_samples: int, seed: int, softening: float) -> tuple[float, float, float]:
        out = np.zeros(3)
        self._check(N.lib.nb_force_error(self._h, int(n_samples), int(seed), float(softening), 0,
                                         N.ptr(out)))
        return float(out[0]), float(out[1]), float(out[2])

    # -- single stages on host arrays ---------------------------------------
    def morton_keys(self, px, py, pz, active, mode: int, cube=None):
        n = len(px)
        px, py, pz = (N.f64a(a, n) for a in (px, py, pz))
        active = N.u8a(active, n)
        keys = np.empty(n, np.uint64)
        idx = np.empty(n, np.int32)
        cube_in = None if cube is None else N.f64a(cube, 4)
        cube_out = np.zeros(4)
        self._check(N.lib.nb_morton_keys(self._h, n, N.ptr(px), N.ptr(py), N.ptr(pz),
                                         N.ptr(active), int(mode), N.ptr(cube_in), N.ptr(keys),
                                         N.ptr(idx), N.ptr(cube_out)))
        return keys, idx, cube_out

    def sort_pairs(self, keys, values):
        keys = np.ascontiguousarray(keys, np.uint64).copy()
        values = np.ascontiguousarray(values, np.int32).copy()
        self._check(N.lib.nb_sort_pairs(self._h, len(keys), N.ptr(keys), N.ptr(values)))
        return keys, values

    def build_octree(self, px, py, pz, mass, active, leaf_capacity: int, cube=None,
                     max_nodes: int | None = None) -> dict:
        n = len(px)
        px, py, pz, mass = (N.f64a(a, n) for a in (px, py, pz, mass))
        active = N.u8a(active, n)
        mx = int(max_nodes) if max_nodes is not None else 2 * max(n, 1)
        nn = np.zeros(1, np.int32)
        o = {k: np.empty(mx, np.int32) for k in ("level", "first_child", "n_children",
                                                   "body_first", "body_count")}
        o["mass"] = np.empty(mx)
        o["com"] = np.empty((mx, 3))
        o["quad"] = np.empty((mx, 6), np.float32)
        sidx = np.empty(n, np.int32)
        skeys = np.empty(n, np.uint64)
        cube_in = None if cube is None else N.f64a(cube, 4)
        self._check(N.lib.nb_build_octree(
            self._h, n, N.ptr(px), N.ptr(py), N.ptr(pz), N.ptr(mass), N.ptr(active),
            N.ptr(cube_in), int(leaf_capacity), mx, N.ptr(nn), N.ptr(o["level"]),
            N.ptr(o["first_child"]), N.ptr(o["n_children"]), N.ptr(o["body_first"]),
            N.ptr(o["body_count"]), N.ptr(o["mass"]), N.ptr(o["com"]), N.ptr(o["quad"]),
            N.ptr(sidx), N.ptr(skeys)))
        k = int(nn[0])
        res = {key: v[:k] for key, v in o.items()}
        res["n_nodes"] = k
        res["sorted_idx"] = sidx
        res["sorted_keys"] = skeys
        return res

    def compact_indices(self, active, mass):
        n = len(active)
        active = N.u8a(active, n)
        mass = N.f64a(mass, n)
        dest = np.empty(n, np.int32)
        kept = np.zeros(1, np.int32)
        self._check(N.lib.nb_compact_indices(self._h, n, N.ptr(active), N.ptr(mass), N.ptr(dest),
                                             N.ptr(kept)))
        return dest, int(kept[0])

    def broad_phase(self, px, py, pz, radius, active, collidable=None, max_pairs: int = 1 << 20):
        n = len(px)
        px, py, pz, radius = (N.f64a(a, n) for a in (px, py, pz, radius))
        active = N.u8a(active, n)
        collidable = None if collidable is None else N.u8a(collidable, n)
        lo = np.empty(max_pairs, np.int32)
        hi = np.empty(max_pairs, np.int32)
        np_ = np.zeros(1, np.int32)
        self._check(N.lib.nb_broad_phase(self._h, n, N.ptr(px), N.ptr(py), N.ptr(pz),
                                         N.ptr(radius), N.ptr(active), N.ptr(collidable),
                                         int(max_pairs), N.ptr(lo), N.ptr(hi), N.ptr(np_)))
        k = int(np_[0])
        return lo[:k].copy(), hi[:k].copy()


    # -- learned MAC ---------------------------------------------------------
    def mac_harvest(self, max_records: int, sample_frac: float, seed: int, softening: float) -> int:
        out = np.zeros(1, np.int32)
        self._check(N.lib.nb_mac_harvest(self._h, int(max_records), float(sample_frac), int(seed),
                                         float(softening), N.ptr(out)))
        return int(out[0])

    def mac_dataset(self):
        n = np.zeros(1, np.int32)
        self._check(N.lib.nb_mac_dataset(self._h, N.ptr(n), None, None))
        X = np.empty((int(n[0]), 8), np.float32)
        Y = np.empty(int(n[0]), np.float32)
        if n[0]:
            self._check(N.lib.nb_mac_dataset(self._h, N.ptr(n), N.ptr(X), N.ptr(Y)))
        return X, Y

    def mac_clear(self):
        self._check(N.lib.nb_mac_clear(self._h))

    def mac_train(self, epochs: int, batch: int = 4096, lr: float = 1e-3, seed: int = 0):
        losses = np.zeros(max(epochs, 1))
        self._check(N.lib.nb_mac_train(self._h, int(epochs), int(batch), float(lr), int(seed),
                                       N.ptr(losses)))
        return losses[:epochs]

    def mac_set_params(self, params: np.ndarray):
        p = np.ascontiguousarray(params, np.float32)
        self._check(N.lib.nb_mac_set_params(self._h, N.ptr(p), len(p)))

    def mac_get_params(self) -> np.ndarray:
        p = np.empty(N.MAC_PARAMS + N.MAC_NORM, np.float32)
        self._check(N.lib.nb_mac_get_params(self._h, N.ptr(p), len(p)))
        return p

    def mac_gradient(self, X, Y):
        X = np.ascontiguousarray(X, np.float32)
        Y = np.ascontiguousarray(Y, np.float32)
        g = np.empty(N.MAC_PARAMS, np.float32)
        loss = np.zeros(1)
        self._check(N.lib.nb_mac_gradient(self._h, N.ptr(X), N.ptr(Y), len(Y), N.ptr(g),
                                          N.ptr(loss)))
        return g, float(loss[0])

    def mac_predict(self, X):
        X = np.ascontiguousarray(X, np.float32)
        y = np.empty(len(X), np.float32)
        self._check(N.lib.nb_mac_predict(self._h, N.ptr(X), len(X), N.ptr(y)))
        return y

    def mac_audit_state(self) -> dict:
        rms, mx = np.zeros(1), np.zeros(1)
        audits, fb = np.zeros(1, np.int64), np.zeros(1, np.int32)
        self._check(N.lib.nb_mac_audit_state(self._h, N.ptr(rms), N.ptr(mx), N.ptr(audits),
                                             N.ptr(fb)))
        return {"rms": float(rms[0]), "max": float(mx[0]), "audits": int(audits[0]),
                "fallback": bool(fb[0])}

    def mac_fit_screen(self):
        self._check(N.lib.nb_mac_fit_screen(self._h))

    def mac_get_screen(self) -> np.ndarray:
        s = np.empty(N.MAC_SCREEN, np.float32)
        self._check(N.lib.nb_mac_get_screen(self._h, N.ptr(s), len(s)))
        return s

    def mac_set_screen(self, screen):
        s = np.ascontiguousarray(screen, np.float32)
        self._check(N.lib.nb_mac_set_screen(self._h, N.ptr(s), len(s)))


class B200PhysicsBackend:
    """IPhysicsComputeBackend + IGravityModelAwareBackend on the B200 engine.

    compute_forces(bodies, softening) fills bodies.ax/ay/az for every row:
    active rows get the sum over active sources, inactive rows 0, as
    CpuParallelBackend.ComputeForces (CpuParallelBackend.cs:69-143).  `mode`
    selects direct (FP32 or FP64) or Barnes-Hut; `theta` is the opening angle
    (BarnesHutBackend.Theta).  last_build_time_ms / last_traversal_time_ms /
    last_total_time_ms mirror BarnesHutBackend.cs:101-107.
    """

    def __init__(self, capacity: int, mode: int = N.MODE_BARNES_HUT, theta: float = 0.5,
                 device: int = 0):
        self.engine = Engine(capacity, device)
        self.mode = mode
        self.theta = theta
        self.enable_shell_theorem = False
        self.use_quadrupole = True
        self.last_build_time_ms = 0.0
        self.last_traversal_time_ms = 0.0
        self.last_total_time_ms = 0.0

    def flags(self) -> int:
        f = self.mode
        if self.enable_shell_theorem:
            f |= N.FLAG_SHELL_THEOREM
        if not self.use_quadrupole:
            f |= N.FLAG_NO_QUADRUPOLE
        return f

    def compute_forces(self, bodies: Bodies, softening: float):
        self.engine.set_param(N.PARAM_THETA, float(self.theta))
        self.engine.compute_forces(bodies.px, bodies.py, bodies.pz, bodies.mass, bodies.active,
                                   softening, self.flags(), radius=bodies.radius,
                                   out=(bodies.ax, bodies.ay, bodies.az))
        t = self.engine.timings()
        self.last_build_time_ms = float(t[N.T_BUILD])
        self.last_traversal_time_ms = float(t[N.T_TRAVERSAL])
        self.last_total_time_ms = float(t[N.T_TOTAL])


class B200SoAIntegrator:
    """ISoAIntegrator ("Verlet-SoA", SoAVerletIntegrator.cs:42-116) running on
    device-resident state: one upload, n steps on the GPU, one download."""

    name = "Verlet-SoA-B200"

    def step(self, bodies: Bodies, backend: B200PhysicsBackend, softening: float, dt: float,
             n_steps: int = 1):
        e = backend.engine
        e.set_param(N.PARAM_THETA, float(backend.theta))
        e.set_state(bodies)
        e.step(n_steps, dt, softening, backend.flags())
        out, _ = e.get_state()
        for k in ("px", "py", "pz", "vx", "vy", "vz", "ax", "ay", "az"):
            getattr(bodies, k)[:] = getattr(out, k)
