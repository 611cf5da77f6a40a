"""Two of the reference's own CUDA kernels, built for sm_100a in place
(oracle/_ref/libcelestial_ref_gpu.so), run on the B200 beside the engine:
the tiled FP64 gravity kernel (engine/src/cuda/gravity_kernel.cu:20-95)
agrees with the FP64 oracle to FP64 rounding (it uses CUDA's rsqrt and FMA
contraction, so not bit for bit), and launch_radix_sort
(engine/src/cuda/morton_kernel.cu:87-230) returns a permutation of its input;
whether that permutation is sorted and stable is recorded by the benchmark's
reference arm, not asserted (its per-pass scatter through a shared-memory
atomicAdd is unstable).  The engine's own sort is compared with the oracle's
stable sort in test_gpu_stages.py."""
from __future__ import annotations

import numpy as np
import pytest

from helpers import rel_err
from nbody_b200 import scenarios

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ref_gpu(oracle):
    if oracle.ref_gpu() is None:
        pytest.skip("oracle/_ref/libcelestial_ref_gpu.so not built")
    return oracle


def test_reference_gravity_kernel_agrees_with_the_oracle(ref_gpu):
    b = scenarios.plummer(1000, 1.0, 1.0, seed=0)
    got, ms = ref_gpu.ref_gpu_gravity(b.px, b.py, b.pz, b.mass, b.active, 1e-4, reps=3)
    want = ref_gpu.direct_forces(b.px, b.py, b.pz, b.mass, b.active, 1e-4)
    assert rel_err(np.array(got), np.array(want)).max() < 1e-12
    assert ms > 0.0


def test_reference_radix_sort_returns_a_permutation(ref_gpu):
    rng = np.random.Generator(np.random.PCG64(5))
    keys = rng.integers(0, 2 ** 63, 100_000, dtype=np.uint64)
    vals = np.arange(100_000, dtype=np.int32)
    k, v, ms = ref_gpu.ref_gpu_radix_sort(keys, vals)
    np.testing.assert_array_equal(np.sort(v), vals)
    np.testing.assert_array_equal(np.sort(k), np.sort(keys))
    np.testing.assert_array_equal(k, keys[v])  # pairs stay together
    assert ms > 0.0
