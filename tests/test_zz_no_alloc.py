"""nb_sort_pairs_noalloc: the sort entry point that allocates no device memory.

It is for callers that cannot call cudaMalloc (their device memory is owned
by their own pool allocator, or they sit on a latency-critical path where a
device-wide synchronising allocation is not allowed).  They pass device
buffers they already own.  This test owns those buffers through torch (the
caller's allocator), calls the entry point through the C ABI twice in a row
on different inputs, and checks each result bit for bit (integer work:
exact) against the existing nb_sort_pairs entry point and against the
oracle's stable sort, which shares no code with the CUDA kernels.

The file is named so that pytest collects it last.
"""
from __future__ import annotations

import numpy as np
import pytest

from nbody_b200 import _native as N

pytestmark = pytest.mark.gpu

MAX_N = 1 << 20  # NB_NOALLOC_SORT_MAX


def _sort_on_device(keys: np.ndarray, vals: np.ndarray):
    import torch

    dk = torch.from_numpy(keys.view(np.int64).copy()).cuda()
    dv = torch.from_numpy(vals.copy()).cuda()
    torch.cuda.synchronize()
    st = N.lib.nb_sort_pairs_noalloc(dk.data_ptr(), dv.data_ptr(), len(keys),
                                     torch.cuda.current_stream().cuda_stream)
    assert st == N.NB_OK, st
    return dk.cpu().numpy().view(np.uint64), dv.cpu().numpy()


def test_noalloc_sort_matches_existing_entry_point_twice(oracle):
    from nbody_b200 import Engine

    rng = np.random.Generator(np.random.PCG64(77))
    cases = [
        rng.integers(0, 2 ** 63, MAX_N, dtype=np.uint64),                  # full size
        rng.integers(0, 97, 300_007).astype(np.uint64) << np.uint64(17),   # many equal keys
    ]
    cases[1][:9] = np.uint64(0xFFFFFFFFFFFFFFFF)
    with Engine(MAX_N) as e:
        for keys in cases:
            vals = np.arange(len(keys), dtype=np.int32)[::-1].copy()
            got_k, got_v = _sort_on_device(keys, vals)
            want_k, want_v = e.sort_pairs(keys, vals)
            np.testing.assert_array_equal(got_k, want_k)
            np.testing.assert_array_equal(got_v, want_v)
            ork, orv = oracle.stable_sort(keys, vals)
            np.testing.assert_array_equal(got_k, ork)
            np.testing.assert_array_equal(got_v, orv)


def test_noalloc_sort_rejects_sizes_beyond_the_maximum():
    st = N.lib.nb_sort_pairs_noalloc(None, None, MAX_N + 1, None)
    assert st == N.NB_ERR_CAPACITY
    assert N.lib.nb_sort_pairs_noalloc(None, None, -1, None) == N.NB_ERR_INVALID_ARG
