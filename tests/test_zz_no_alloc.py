"""RadixSortNoAlloc against RadixSort, through the C ABI, on a GPU.

RadixSortNoAlloc exists for callers that cannot allocate device memory (a
host loop whose own pool allocator owns the GPU's memory, or a
latency-critical loop that must not pay a first-call allocation).  It keeps
its scratch in a fixed device array inside the library.  This file is
collected last so that a run stopping at the first failure has already run
every other test; it also passes when run alone in a fresh process.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _keys(n, bits, seed):
    rng = np.random.default_rng(seed)
    kv = np.empty(2 * n, dtype=np.uint32)
    hi = min(2 ** bits, 1 << 32)
    kv[0::2] = rng.integers(0, hi, n, dtype=np.uint64).astype(np.uint32)
    kv[0::2][::7] = 4242 % hi          # ties, to check stability
    kv[1::2] = rng.permutation(n).astype(np.uint32)
    return kv


def test_no_alloc_sort_matches_allocating_sort_on_two_calls(dem, cuda):
    torch = cuda
    # two calls in a row; the second reuses the array the first left behind
    for n, bits, seed in ((300_001, 32, 11), (1_000_003, 20, 12)):
        kv = _keys(n, bits, seed)
        a0 = torch.from_numpy(kv.view(np.int32).copy()).cuda()
        a1 = torch.zeros_like(a0)
        b0 = torch.from_numpy(kv.view(np.int32).copy()).cuda()
        b1 = torch.zeros_like(b0)
        dem.compat.RadixSort(a0, a1, n, bits)
        dem.compat.RadixSortNoAlloc(b0, b1, n, bits)
        torch.cuda.synchronize()
        got = b0.cpu().numpy().view(np.uint32)
        np.testing.assert_array_equal(got, a0.cpu().numpy().view(np.uint32))   # integer result: bit-exact
        assert np.all(np.diff(got[0::2].astype(np.int64)) >= 0)


def test_no_alloc_sort_at_its_limit_is_the_stable_order_and_allocates_nothing(dem, cuda):
    """Exactly 4,194,304 records (the fixed array at its fullest), twice: the
    result is numpy's stable order of the keys, and the second call leaves
    the device's free memory unchanged (the first may load the library's
    device code, which is why a caller makes it during set-up)."""
    torch = cuda
    n, bits = 1 << 22, 24
    kv = _keys(n, bits, 21)
    order = np.argsort(kv[0::2], kind="stable")
    want = np.empty_like(kv)
    want[0::2], want[1::2] = kv[0::2][order], kv[1::2][order]
    d0 = torch.from_numpy(kv.view(np.int32).copy()).cuda()
    d1 = torch.zeros_like(d0)
    dem.compat.RadixSortNoAlloc(d0, d1, n, bits)          # set-up call
    torch.cuda.synchronize()
    np.testing.assert_array_equal(d0.cpu().numpy().view(np.uint32), want)
    d0.copy_(torch.from_numpy(kv.view(np.int32).copy()))
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    dem.compat.RadixSortNoAlloc(d0, d1, n, bits)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    np.testing.assert_array_equal(d0.cpu().numpy().view(np.uint32), want)


def test_no_alloc_sort_rejects_sizes_above_its_limit(dem, cuda):
    with pytest.raises(dem.DemError) as ei:
        dem.compat.RadixSortNoAlloc(0, 0, (1 << 22) + 1, 32)
    assert ei.value.code == dem.DEM_ERR_ARG
    assert "4194304" in str(ei.value)
