"""ctypes binding of libnbody_b200.so (declarations in include/nbody_b200.h).

The library is loaded from the package directory.  There is no fallback:
if it is missing or cannot be loaded, importing this module raises.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent.parent / "libnbody_b200.so"

if not LIB_PATH.exists():
    raise ImportError(f"{LIB_PATH} is missing: run celestial-mechanics-desktop_b200/build.py")
lib = C.CDLL(str(LIB_PATH))

# status codes
NB_OK = 0
NB_ERR_INVALID_ARG = -1
NB_ERR_CAPACITY = -2
NB_ERR_CUDA = -3
NB_ERR_TIMEOUT = -4
NB_ERR_STACK_OVERFLOW = -5
NB_ERR_NO_DEVICE = -6
NB_ERR_NONFINITE = -7
NB_ERR_STATE = -8
# modes / flags
MODE_DIRECT = 0
MODE_DIRECT_FP64 = 1
MODE_BARNES_HUT = 2
MODE_BARNES_HUT_REF = 3
FLAG_SHELL_THEOREM = 0x10
FLAG_NO_QUADRUPOLE = 0x20
FLAG_COLLISIONS = 0x40
FLAG_LEARNED_MAC = 0x80
FLAG_YOSHIDA4 = 0x100
FLAG_ADAPTIVE_DT = 0x200
FLAG_ORDER_SIMD = 0x400
FLAG_ORDER_PAIRWISE = 0x800
# parameters
PARAM_THETA = 1
PARAM_LEAF_CAPACITY = 2
PARAM_MAX_MERGES_FRAME = 3
PARAM_MAX_MERGES_BODY = 4
PARAM_MIN_RADIUS = 5
PARAM_DENSITY_MERGE = 6
PARAM_TIMING = 7
PARAM_MAC_BUDGET = 8
PARAM_GROUP_BODIES = 9
PARAM_GROUP_PACK = 10
PARAM_MAC_THETA_LO = 11
PARAM_MAC_THETA_HI = 12
PARAM_MAC_SCREEN_QUANTILE = 13
PARAM_ENS_DIRECT_SHAPE = 14
PARAM_MAC_AUDIT_INTERVAL = 15
PARAM_MAC_AUDIT_SAMPLES = 16
PARAM_MAC_AUDIT_RMS = 17
PARAM_ADAPTIVE_ETA = 18
PARAM_ADAPTIVE_DT_MIN = 19
PARAM_ADAPTIVE_DT_MAX = 20
PARAM_GROUP_SPAN = 21
PARAM_ENS_WALK_SHAPE = 22
# nb_ens_autotune_tree choices: (walk block shape, walk-group span)
# (walk block shape, walk-group span, bodies per group) of each tree autotune choice
ENS_TREE_CHOICES = ([(w, sp, 32) for w in (0, 1) for sp in (0, 256, 512, 1024)] +
                    [(0, sp, 64) for sp in (256, 512, 1024)])
ENS_SHAPES = [(64, 1), (64, 2), (64, 4), (128, 1), (128, 2), (128, 4), (256, 1), (256, 2), (256, 4)]
# timings / counters
T_BUILD, T_TRAVERSAL, T_TOTAL, T_SORT, T_TREE, T_COLLIDE, T_COUNT = range(7)
(C_CELL_INTERACTIONS, C_BODY_INTERACTIONS, C_NODES, C_ACTIVE, C_PAIRS, C_MERGES, C_OVERFLOWS, C_GROUPS,
 C_MAX_GROUP_WORK, C_MAC_EVALS, C_MAC_AUDITS, C_MAC_FALLBACK, C_COUNT) = range(13)

vp = C.c_void_p
i32 = C.c_int32
f64 = C.c_double
u64 = C.c_uint64
P = C.c_void_p  # every array argument is passed as a raw pointer

_SIGS = {
    "nb_create": (i32, [i32, i32, C.POINTER(vp)]),
    "nb_destroy": (i32, [vp]),
    "nb_last_error": (C.c_char_p, [vp]),
    "nb_set_param_f64": (i32, [vp, i32, f64]),
    "nb_set_param_i32": (i32, [vp, i32, i32]),
    "nb_get_timings": (i32, [vp, P, i32]),
    "nb_get_counters": (i32, [vp, P, i32]),
    "nb_get_adaptive_dt": (i32, [vp, P]),
    "nb_max_acceleration": (i32, [vp, P]),
    "nb_get_body_count": (i32, [vp, P, P]),
    "nb_stream": (vp, [vp]),
    "nb_version": (C.c_char_p, []),
    "nb_compute_forces": (i32, [vp, i32, P, P, P, P, P, P, f64, i32, P, P, P]),
    "nb_set_state": (i32, [vp, i32, P, P, P, P, P, P, P, P, P, P, P, P, P, P]),
    "nb_get_state": (i32, [vp, P, P, P, P, P, P, P, P, P, P, P, P, P, P]),
    "nb_step": (i32, [vp, i32, f64, f64, i32]),
    "nb_diagnostics": (i32, [vp, f64, i32, P]),
    "nb_force_error": (i32, [vp, i32, u64, f64, i32, P]),
    "nb_morton_keys": (i32, [vp, i32, P, P, P, P, i32, P, P, P, P]),
    "nb_sort_pairs": (i32, [vp, i32, P, P]),
    "nb_sort_pairs_noalloc": (i32, [P, P, i32, vp]),
    "nb_build_octree": (i32, [vp, i32, P, P, P, P, P, P, i32, i32, P, P, P, P, P, P, P, P, P,
                              P, P]),
    "nb_compact_indices": (i32, [vp, i32, P, P, P, P]),
    "nb_broad_phase": (i32, [vp, i32, P, P, P, P, P, P, i32, P, P, P]),
    "nb_mac_harvest": (i32, [vp, i32, f64, u64, f64, P]),
    "nb_mac_dataset": (i32, [vp, P, P, P]),
    "nb_mac_clear": (i32, [vp]),
    "nb_mac_train": (i32, [vp, i32, i32, f64, u64, P]),
    "nb_mac_set_params": (i32, [vp, P, i32]),
    "nb_mac_get_params": (i32, [vp, P, i32]),
    "nb_mac_gradient": (i32, [vp, P, P, i32, P, P]),
    "nb_mac_predict": (i32, [vp, P, i32, P]),
    "nb_mac_fit_screen": (i32, [vp]),
    "nb_mac_audit_state": (i32, [vp, P, P, P, P]),
    "nb_mac_get_screen": (i32, [vp, P, i32]),
    "nb_mac_set_screen": (i32, [vp, P, i32]),
    "nb_ens_create": (i32, [i32, P, i32, i32, C.POINTER(vp)]),
    "nb_ens_destroy": (i32, [vp]),
    "nb_ens_last_error": (C.c_char_p, [vp]),
    "nb_ens_info": (i32, [vp, P, i32]),
    "nb_ens_set_param_f64": (i32, [vp, i32, f64]),
    "nb_ens_set_param_i32": (i32, [vp, i32, i32]),
    "nb_ens_set_state": (i32, [vp, P, P, P, P, P, P, P]),
    "nb_ens_get_state": (i32, [vp, P, P, P, P, P, P, P, P, P]),
    "nb_ens_compute_forces": (i32, [vp, f64]),
    "nb_ens_step": (i32, [vp, i32, f64, f64]),
    "nb_ens_autotune": (i32, [vp, f64, P, P]),
    "nb_ens_autotune_tree": (i32, [vp, f64, P, P]),
    "nb_ens_force_error": (i32, [vp, i32, u64, f64, P, P]),
    "nb_ens_energy": (i32, [vp, f64, P, P, P]),
    "nb_ens_get_counters": (i32, [vp, P, i32]),
    "nb_ens_get_timings": (i32, [vp, P]),
}
MAC_PARAMS = 4801
MAC_NORM = 18
MAC_SCREEN = 10
for _name, (_res, _args) in _SIGS.items():
    _f = getattr(lib, _name)
    _f.restype = _res
    _f.argtypes = _args

EXPORTED = tuple(_SIGS)


def ptr(a):
    """Raw data pointer of a C-contiguous numpy array (None passes NULL)."""
    if a is None:
        return None
    if not a.flags["C_CONTIGUOUS"]:
        raise ValueError("arrays must be C-contiguous")
    return a.ctypes.data


def f64a(a, n=None):
    a = np.ascontiguousarray(a, dtype=np.float64)
    if n is not None and a.shape != (n,):
        raise ValueError(f"expected shape ({n},), got {a.shape}")
    return a


def u8a(a, n=None):
    a = np.ascontiguousarray(a, dtype=np.uint8)
    if n is not None and a.shape != (n,):
        raise ValueError(f"expected shape ({n},), got {a.shape}")
    return a
