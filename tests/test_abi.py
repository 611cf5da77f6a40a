"""The C-ABI library loads and exports every symbol include/nbody_b200.h
declares; host-side argument checks.  No GPU compute calls.  CPU only."""
from __future__ import annotations

import ctypes as C
import re
import subprocess
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "nbody_b200.h"


def declared_symbols():
    return sorted(set(re.findall(r"NB_API\s+[\w\s\*]+?\b(nb_\w+)\s*\(", HEADER.read_text())))


def test_library_exports_every_declared_symbol():
    from nbody_b200 import _native as N

    syms = declared_symbols()
    assert len(syms) >= 20
    for s in syms:
        assert hasattr(N.lib, s), s
    nm = subprocess.run(["nm", "-D", "--defined-only", str(N.LIB_PATH)], capture_output=True,
                        text=True, check=True).stdout
    exported = set(re.findall(r"\sT\s(nb_\w+)", nm))
    assert set(syms) <= exported
    # nothing beyond the header leaks out of the library
    assert exported <= set(syms)
    assert set(N.EXPORTED) == set(syms)


def test_version_string():
    from nbody_b200 import _native as N

    assert b"sm_100a" in N.lib.nb_version()


def test_null_and_bad_arguments_rejected_without_device():
    from nbody_b200 import _native as N

    h = C.c_void_p()
    assert N.lib.nb_create(0, 0, C.byref(h)) == N.NB_ERR_INVALID_ARG
    assert N.lib.nb_create(16, 0, None) == N.NB_ERR_INVALID_ARG
    assert N.lib.nb_destroy(None) == N.NB_ERR_INVALID_ARG
    assert N.lib.nb_step(None, 1, 1e-3, 1e-4, 0) == N.NB_ERR_INVALID_ARG
    out = np.zeros(3)
    assert N.lib.nb_get_timings(None, out.ctypes.data, 3) == N.NB_ERR_INVALID_ARG


def test_no_device_is_reported_not_faked():
    """Without a CUDA device nb_create must fail with NB_ERR_NO_DEVICE:
    there is no CPU fallback."""
    import torch

    from nbody_b200 import _native as N

    if torch.cuda.is_available():
        return
    h = C.c_void_p()
    assert N.lib.nb_create(1024, 0, C.byref(h)) == N.NB_ERR_NO_DEVICE
    assert not h.value
