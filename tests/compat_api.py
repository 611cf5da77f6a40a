"""ctypes signatures of the `celestial_*` compatibility functions
(include/celestial_compat.h), shared by the CPU and GPU tests."""
from __future__ import annotations

import ctypes as C
import re
from pathlib import Path

HEADER = Path(__file__).resolve().parent.parent / "include" / "celestial_compat.h"

P = C.c_void_p
i32, f64, u32 = C.c_int32, C.c_double, C.c_uint32


class CelestialVersion(C.Structure):
    _fields_ = [("major", i32), ("minor", i32), ("patch", i32)]


SIGS = {
    "celestial_init": (i32, [i32]),
    "celestial_shutdown": (None, []),
    "celestial_set_particles": (None, [P] * 12 + [i32]),
    "celestial_get_accelerations": (None, [P, P, P, i32]),
    "celestial_get_positions": (None, [P, P, P, i32]),
    "celestial_get_velocities": (None, [P, P, P, i32]),
    "celestial_compute_forces": (None, [f64]),
    "celestial_step": (None, [f64, f64]),
    "celestial_update": (i32, [f64]),
    "celestial_set_compute_mode": (None, [i32]),
    "celestial_set_theta": (None, [f64]),
    "celestial_set_dt": (None, [f64]),
    "celestial_set_softening": (None, [f64]),
    "celestial_set_integrator": (None, [i32]),
    "celestial_get_integrator": (i32, []),
    "celestial_set_adaptive_timestep": (None, [i32, f64, f64, f64, f64]),
    "celestial_get_adaptive_dt": (f64, []),
    "celestial_is_adaptive_dt_enabled": (i32, []),
    "celestial_compute_energy_snapshot": (None, []),
    "celestial_get_energy_drift": (f64, []),
    "celestial_get_momentum_drift": (f64, []),
    "celestial_get_angular_momentum_drift": (f64, []),
    "celestial_get_accumulated_error": (f64, []),
    "celestial_get_last_gpu_time_ms": (f64, []),
    "celestial_get_last_tree_build_ms": (f64, []),
    "celestial_get_last_tree_traverse_ms": (f64, []),
    "celestial_get_particle_count": (i32, []),
    "celestial_get_active_particle_count": (i32, []),
    "celestial_get_last_merge_count": (i32, []),
    "celestial_set_collision_mode": (None, [i32]),
    "celestial_set_max_merges_per_frame": (None, [i32]),
    "celestial_set_max_merges_per_body": (None, [i32]),
    "celestial_set_density_preserving_merge": (None, [i32]),
    "celestial_api_version": (CelestialVersion, []),
    "celestial_query_capabilities": (u32, []),
    "celestial_get_last_error_message": (C.c_char_p, []),
}


def declared():
    return sorted(set(re.findall(r"NB_API\s+[\w\s\*]+?\b(celestial_\w+)\s*\(", HEADER.read_text())))


def bind(lib):
    for name, (res, args) in SIGS.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib
