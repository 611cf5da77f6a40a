"""Batched ensembles of independent systems (nb_ens_* in include/nbody_b200.h).

No reference counterpart: the reference integrates one system per
NBodySolver.Step.  `Ensemble` owns one handle; arrays are the systems'
bodies concatenated in the order of `sizes`.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N
from .engine import NBodyError
from .scenarios import Bodies


class Ensemble:
    def __init__(self, sizes, ds_max_n: int = 2048, device: int = 0):
        self.sizes = np.ascontiguousarray(sizes, np.int32)
        h = C.c_void_p()
        st = N.lib.nb_ens_create(len(self.sizes), N.ptr(self.sizes), int(ds_max_n), int(device),
                                 C.byref(h))
        if st != N.NB_OK:
            raise NBodyError(st, "nb_ens_create failed")
        self._h = h
        self.n = int(self.sizes.sum())
        self.offsets = np.concatenate([[0], np.cumsum(self.sizes)]).astype(np.int64)

    def close(self):
        if getattr(self, "_h", None):
            N.lib.nb_ens_destroy(self._h)
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
            msg = N.lib.nb_ens_last_error(self._h)
            raise NBodyError(st, msg.decode() if msg else "")

    def info(self) -> dict:
        out = np.zeros(6, np.int64)
        self._check(N.lib.nb_ens_info(self._h, N.ptr(out), 6))
        keys = ("systems", "direct_systems", "tree_systems", "bodies", "direct_bodies",
                "tree_bodies")
        return {k: int(v) for k, v in zip(keys, out)}

    def set_param(self, param: int, value):
        if isinstance(value, float):
            self._check(N.lib.nb_ens_set_param_f64(self._h, param, value))
        else:
            self._check(N.lib.nb_ens_set_param_i32(self._h, param, int(value)))

    def set_state(self, systems: list[Bodies]):
        if len(systems) != len(self.sizes) or any(b.n != k for b, k in zip(systems, self.sizes)):
            raise ValueError("systems do not match the ensemble's sizes")
        cat = {k: np.ascontiguousarray(np.concatenate([getattr(b, k) for b in systems]),
                                       np.float64)
               for k in ("px", "py", "pz", "vx", "vy", "vz", "mass")}
        self._check(N.lib.nb_ens_set_state(self._h, *(N.ptr(cat[k]) for k in
                                                       ("px", "py", "pz", "vx", "vy", "vz",
                                                        "mass"))))

    def get_state(self) -> dict:
        keys = ("px", "py", "pz", "vx", "vy", "vz", "ax", "ay", "az")
        out = {k: np.empty(self.n) for k in keys}
        self._check(N.lib.nb_ens_get_state(self._h, *(N.ptr(out[k]) for k in keys)))
        return out

    def compute_forces(self, softening: float):
        self._check(N.lib.nb_ens_compute_forces(self._h, float(softening)))

    def step(self, n_steps: int, dt: float, softening: float):
        self._check(N.lib.nb_ens_step(self._h, int(n_steps), float(dt), float(softening)))

    def autotune(self, softening: float):
        shape = np.zeros(1, np.int32)
        ms = np.zeros(len(N.ENS_SHAPES))
        self._check(N.lib.nb_ens_autotune(self._h, float(softening), N.ptr(shape), N.ptr(ms)))
        return int(shape[0]), ms

    def autotune_tree(self, softening: float):
        """Fastest (walk block shape, walk-group span) of the tree branch on
        the current state; returns (choice index into N.ENS_TREE_CHOICES,
        ms per choice, -1 for choices not tried)."""
        choice = np.zeros(1, np.int32)
        ms = np.zeros(len(N.ENS_TREE_CHOICES))
        self._check(N.lib.nb_ens_autotune_tree(self._h, float(softening), N.ptr(choice),
                                               N.ptr(ms)))
        return int(choice[0]), ms

    def force_error(self, samples: int, seed: int, softening: float):
        rms = np.zeros(len(self.sizes))
        mx = np.zeros(len(self.sizes))
        self._check(N.lib.nb_ens_force_error(self._h, int(samples), int(seed), float(softening),
                                             N.ptr(rms), N.ptr(mx)))
        return rms, mx

    def energy(self, softening: float):
        e = np.zeros(len(self.sizes))
        ke = np.zeros(len(self.sizes))
        pe = np.zeros(len(self.sizes))
        self._check(N.lib.nb_ens_energy(self._h, float(softening), N.ptr(e), N.ptr(ke), N.ptr(pe)))
        return e, ke, pe

    def counters(self) -> dict:
        out = np.zeros(6, np.int64)
        self._check(N.lib.nb_ens_get_counters(self._h, N.ptr(out), 6))
        keys = ("direct_pairs", "tree_cell", "tree_body", "graph_launches", "direct_items",
                "direct_shape")
        return {k: int(v) for k, v in zip(keys, out)}

    def ms_per_step(self) -> float:
        out = np.zeros(1)
        self._check(N.lib.nb_ens_get_timings(self._h, N.ptr(out)))
        return float(out[0])
