"""The allocation-free radix sort entry point, through the C ABI.

gs_radix_sort_pairs_noalloc serves callers that cannot let the library
allocate device memory (a host that owns all device memory, a loop that must
not pay an allocation's latency or implicit synchronisation, a binding that
forbids hidden allocations). Its scratch is a fixed device array for at most
1,048,576 pairs. Two calls in a row must each give exactly the result of the
allocating gs_radix_sort_pairs on the same input (integer sort: exact), and an
oversized input must be rejected.

This file sorts last in collection order so that a run stopping at the first
failure has already run every other test; it also passes on its own in a
fresh process.
"""
import numpy as np
import pytest

from splattar_b200 import GsError
from splattar_b200.rasterizer import radix_sort_pairs, radix_sort_pairs_noalloc

pytestmark = pytest.mark.gpu

MAX_PAIRS = 1 << 20


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).cuda()


def _host(t):
    return t.cpu().numpy().view(np.uint32)


def _both(keys, vals, key_bits):
    import torch
    n = keys.size
    ka, va = _dev(keys), _dev(vals)
    radix_sort_pairs(ka.data_ptr(), va.data_ptr(), n, key_bits)
    kb, vb = _dev(keys), _dev(vals)
    radix_sort_pairs_noalloc(kb.data_ptr(), vb.data_ptr(), n, key_bits)
    torch.cuda.synchronize()
    return (_host(ka), _host(va)), (_host(kb), _host(vb))


def test_noalloc_sort_matches_allocating_sort_twice():
    rng = np.random.default_rng(20)
    cases = [
        # heavy duplicates on 13 bits (two passes), odd size
        ((rng.integers(0, 8192, 1_000_003)).astype(np.uint32), 13),
        # full-range 32-bit keys (four passes), the maximum size
        (rng.integers(0, 2**32, MAX_PAIRS, dtype=np.uint64).astype(np.uint32), 32),
        # odd pass counts (three passes, one pass): the sorted pairs end in the
        # scratch array and are copied back into the caller's arrays
        ((rng.integers(0, 2**24, 777_777)).astype(np.uint32), 24),
        ((rng.integers(0, 32, 4099)).astype(np.uint32), 5),
    ]
    for keys, bits in cases:  # two calls in a row, the second reusing the scratch
        vals = np.arange(keys.size, dtype=np.uint32)
        (ka, va), (kb, vb) = _both(keys, vals, bits)
        assert np.array_equal(ka, kb) and np.array_equal(va, vb)
        order = np.argsort(keys, kind="stable")
        assert np.array_equal(kb, keys[order]) and np.array_equal(vb, vals[order])


def test_noalloc_sort_rejects_oversized_input():
    import torch
    n = MAX_PAIRS + 1
    k = torch.zeros(n, dtype=torch.int32, device="cuda")
    v = torch.zeros(n, dtype=torch.int32, device="cuda")
    with pytest.raises(GsError, match="GS_ERR_CAPACITY"):
        radix_sort_pairs_noalloc(k.data_ptr(), v.data_ptr(), n, 32)
