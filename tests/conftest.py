"""Shared test setup: import paths, the gpu marker, fixtures."""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
PKG_DIR = ROOT / "celestial-mechanics-desktop_b200"
for p in (str(PKG_DIR), str(ROOT / "oracle"), str(ROOT)):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) GPU and the built engine")


def bodies_dict(b) -> dict:
    """Bodies dataclass -> the dict the oracle wrappers take."""
    d = {k: v for k, v in b.__dict__.items()}
    if d.get("density") is None:
        d["density"] = np.zeros(b.n)
    return d


@pytest.fixture(scope="session")
def oracle():
    import oracle as o  # noqa: WPS433

    o.lib()
    return o


@pytest.fixture(scope="session")
def ref_lib(oracle):
    if oracle.ref() is None:
        pytest.skip("oracle/_ref not built (reference tree absent at build time)")
    return oracle


@pytest.fixture(scope="session")
def engine():
    from nbody_b200 import Engine

    e = Engine(1 << 21)
    yield e
    e.close()
