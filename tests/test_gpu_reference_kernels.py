"""The reference's own CUDA paths, built for sm_100a in place
(oracle/_ref/libcelestial_ref_gpu.so), run on the B200 beside the engine:
the tiled FP64 gravity kernel (engine/src/cuda/gravity_kernel.cu:20-95)
agrees with the FP64 oracle to FP64 rounding (it uses CUDA's rsqrt and FMA
contraction, so not bit for bit), and launch_radix_sort
(engine/src/cuda/morton_kernel.cu:87-230) returns a permutation of its input;
whether that permutation is sorted and stable is recorded by the benchmark's
reference arm, not asserted (its per-pass scatter through a shared-memory
atomicAdd is unstable).  The engine's own sort is compared with the oracle's
stable sort in test_gpu_stages.py.  GpuTreeSolver::compute_forces
(engine/src/cuda/gpu_tree.cu:112-193) gives theta-0.5 monopole forces: its
error against the FP64 direct sum is that of the reference's CPU
BarnesHutSolver to within 20 %."""
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


def test_reference_gpu_tree_solver_forces(ref_gpu):
    b = scenarios.plummer(20_000, 1.0, 1.0, seed=3)
    got, ms, build, trav = ref_gpu.ref_gpu_tree(b.px, b.py, b.pz, b.mass, b.active, 1e-4, 0.5,
                                                reps=1)
    assert ms > 0.0 and build >= 0.0 and trav >= 0.0
    rows = np.arange(0, 20_000, 7, dtype=np.int32)
    want = ref_gpu.direct_forces_targets(b.px, b.py, b.pz, b.mass, b.active, 1e-4, rows)
    e_gpu = ref_gpu.force_error((got[0][rows], got[1][rows], got[2][rows]), want)[2]
    cpu = ref_gpu.ref_bh_forces(b.px, b.py, b.pz, b.mass, b.active, 1e-4, 0.5, True, 4)[0]
    e_cpu = ref_gpu.force_error((cpu[0][rows], cpu[1][rows], cpu[2][rows]), want)[2]
    assert 0.0 < e_gpu < 1e-2
    assert e_gpu == pytest.approx(e_cpu, rel=0.2)
