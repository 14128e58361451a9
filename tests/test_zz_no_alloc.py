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


def test_no_alloc_sort_rejects_sizes_above_its_limit(dem, cuda):
    with pytest.raises(dem.DemError) as ei:
        dem.compat.RadixSortNoAlloc(0, 0, (1 << 22) + 1, 32)
    assert ei.value.code == dem.DEM_ERR_ARG
    assert "4194304" in str(ei.value)
