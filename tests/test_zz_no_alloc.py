"""bz_sort_pairs_noalloc, the allocation-free sort for callers that may not allocate device
memory (hosts that reserve HBM for their own pool or arena, step loops that cannot afford
cudaMalloc/cudaFree), checked against the engine's own allocating path.

bz_morton_keys sorts the Morton keys of an engine's state and returns the sorted keys and the
stable permutation.  Feeding the same keys, unsorted, with values 0..n-1 through the
allocation-free sort must reproduce both exactly (integer work: bit-exact).  Two calls in a
row, on different data and sizes, check that the shared scratch array left by one call does
not disturb the next.  This file sorts last so that a run stopping at the first failure has
already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import plummer

pytestmark = pytest.mark.gpu


def _engine_order(n, seed):
    from blitzar_b200._lib import Engine

    pos = plummer(n, seed)
    m = np.full(n, 1.0 / n, np.float32)
    with Engine(n, solver=0) as e:
        e.set_state(pos, None, m)
        keys, perm = e.morton_keys()
    unsorted = np.empty_like(keys)
    unsorted[perm] = keys
    return unsorted, keys, perm


def _noalloc_sort(L, keys_host, bits=64):
    import torch

    n = len(keys_host)
    k = torch.from_numpy(keys_host.view(np.int64)).cuda()
    v = torch.arange(n, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    st = L.bz_sort_pairs_noalloc(C.c_void_p(k.data_ptr()), C.c_void_p(v.data_ptr()), n, bits, 0)
    return st, k.cpu().numpy().view(np.uint64), v.cpu().numpy()


def test_noalloc_sort_matches_engine_two_calls(gpu):
    from blitzar_b200._lib import BZ_OK

    L = gpu
    # call 1: ragged last tile; call 2: the stated maximum size, different data
    for n, seed in ((300_001, 11), (1 << 20, 12)):
        unsorted, ref_keys, ref_perm = _engine_order(n, seed)
        st, keys, vals = _noalloc_sort(L, unsorted)
        assert st == BZ_OK
        assert np.array_equal(keys, ref_keys)
        assert np.array_equal(vals, ref_perm)


def test_noalloc_sort_rejects_sizes_beyond_maximum(gpu):
    from blitzar_b200._lib import BZ_INVALID_ARGUMENT, BZ_OK

    L = gpu
    assert L.bz_sort_pairs_noalloc(None, None, (1 << 20) + 1, 64, 0) == BZ_INVALID_ARGUMENT
    assert L.bz_sort_pairs_noalloc(None, None, 1000, 12, 0) == BZ_INVALID_ARGUMENT
    assert L.bz_sort_pairs_noalloc(None, None, 0, 64, 0) == BZ_OK
