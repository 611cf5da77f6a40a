"""B200 (sm_100a) N-body force engine: Python host layer.

The compute path is libnbody_b200.so (CUDA, include/nbody_b200.h); this
package only binds it.  The library is loaded the first time anything but
the scenario generators (``nbody_b200.scenarios``, ``Bodies``) is used, and
that load raises if it is missing: there is no CPU fallback.  Generating
inputs alone (as a CPU baseline does) therefore maps no engine code.
"""
from __future__ import annotations

import importlib

from .scenarios import Bodies  # noqa: F401  (pure numpy)

# names served by the modules that load libnbody_b200.so
_LAZY = {
    "native": ("._native", None),
    "FLAG_ADAPTIVE_DT": ("._native", "FLAG_ADAPTIVE_DT"),
    "FLAG_COLLISIONS": ("._native", "FLAG_COLLISIONS"),
    "FLAG_LEARNED_MAC": ("._native", "FLAG_LEARNED_MAC"),
    "FLAG_NO_QUADRUPOLE": ("._native", "FLAG_NO_QUADRUPOLE"),
    "FLAG_YOSHIDA4": ("._native", "FLAG_YOSHIDA4"),
    "FLAG_SHELL_THEOREM": ("._native", "FLAG_SHELL_THEOREM"),
    "FLAG_ORDER_SIMD": ("._native", "FLAG_ORDER_SIMD"),
    "FLAG_ORDER_PAIRWISE": ("._native", "FLAG_ORDER_PAIRWISE"),
    "MODE_BARNES_HUT": ("._native", "MODE_BARNES_HUT"),
    "MODE_BARNES_HUT_REF": ("._native", "MODE_BARNES_HUT_REF"),
    "MODE_DIRECT": ("._native", "MODE_DIRECT"),
    "MODE_DIRECT_FP64": ("._native", "MODE_DIRECT_FP64"),
    "Engine": (".engine", "Engine"),
    "NBodyError": (".engine", "NBodyError"),
    "B200PhysicsBackend": (".engine", "B200PhysicsBackend"),
    "B200SoAIntegrator": (".engine", "B200SoAIntegrator"),
    "Ensemble": (".ensemble", "Ensemble"),
}


def __getattr__(name):
    try:
        mod, attr = _LAZY[name]
    except KeyError:
        raise AttributeError(f"module 'nbody_b200' has no attribute {name!r}") from None
    m = importlib.import_module(mod, __name__)
    value = m if attr is None else getattr(m, attr)
    globals()[name] = value
    return value


__all__ = ["Engine", "Ensemble", "NBodyError", "B200PhysicsBackend", "B200SoAIntegrator",
           "Bodies"]
