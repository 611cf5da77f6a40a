"""The `celestial_*` compatibility layer on the CPU: every function
include/celestial_compat.h declares is exported (and no other celestial_
symbol), and without a GPU it behaves as the reference's API does without
an engine: init reports the missing device, everything else is a no-op."""
from __future__ import annotations

import re
import subprocess

import compat_api as A


def test_compat_exports_every_declared_function():
    from nbody_b200 import _native as N

    syms = A.declared()
    assert len(syms) == len(A.SIGS) and set(syms) == set(A.SIGS)
    nm = subprocess.run(["nm", "-D", "--defined-only", str(N.LIB_PATH)], capture_output=True,
                        text=True, check=True).stdout
    exported = set(re.findall(r"\sT\s(celestial_\w+)", nm))
    assert exported == set(syms)


def test_compat_without_device():
    import torch

    from nbody_b200 import _native as N

    if torch.cuda.is_available():
        return  # the GPU tests cover this path with a device
    lib = A.bind(N.lib)
    assert lib.celestial_init(16) == -5  # DeviceNotFound
    assert b"nb_create" in lib.celestial_get_last_error_message()
    # no engine: calls return the reference's neutral values
    assert lib.celestial_get_particle_count() == 0
    assert lib.celestial_update(1.0) == 0
    assert lib.celestial_get_energy_drift() == 0.0
    lib.celestial_step(1e-3, 1e-4)
    lib.celestial_shutdown()
    v = lib.celestial_api_version()
    assert (v.major, v.minor, v.patch) == (1, 0, 0)
    caps = lib.celestial_query_capabilities()
    assert caps & (1 << 2) and caps & (1 << 6) and not caps & (1 << 3)  # Yoshida4, adaptive; no PN
