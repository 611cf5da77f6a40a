"""B200 (sm_100a) N-body force engine: Python host layer.

The compute path is libnbody_b200.so (CUDA, include/nbody_b200.h); this
package only binds it.  Importing it loads the library and raises if it is
missing: there is no CPU fallback.
"""
from . import _native as native  # noqa: F401  (loads the library)
from ._native import (FLAG_ADAPTIVE_DT, FLAG_COLLISIONS, FLAG_LEARNED_MAC,  # noqa: F401
                      FLAG_NO_QUADRUPOLE, FLAG_YOSHIDA4,
                      FLAG_SHELL_THEOREM, MODE_BARNES_HUT, MODE_BARNES_HUT_REF, MODE_DIRECT,
                      MODE_DIRECT_FP64)
from .engine import B200PhysicsBackend, B200SoAIntegrator, Engine, NBodyError  # noqa: F401
from .ensemble import Ensemble  # noqa: F401
from .scenarios import Bodies  # noqa: F401

__all__ = ["Engine", "Ensemble", "NBodyError", "B200PhysicsBackend", "B200SoAIntegrator",
           "Bodies"]
