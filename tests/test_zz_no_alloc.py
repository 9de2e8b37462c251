"""GPU test of brt_radix_sort_pairs_noalloc, the sort entry point that
allocates nothing (for callers that cannot call cudaMalloc: frame loops that
must not stall the device, code under another framework's allocator, hosts
with a fixed memory budget).  Its scratch is a static device array shared by
every call, so two calls in a row must not see each other's leftovers.

It is compared with the allocating entry point brt_radix_sort_pairs (integer
sort: the results must be identical).  The file name makes pytest collect it
last; it also passes alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

from behavert_b200 import _abi, radix_sort_pairs, radix_sort_scratch_bytes

pytestmark = pytest.mark.gpu


def _noalloc(din, dout, n, bits):
    st = _abi.lib().brt_radix_sort_pairs_noalloc(_abi.ptr(din), _abi.ptr(dout), n, bits, None)
    _abi.check(st, "brt_radix_sort_pairs_noalloc")


def _pairs(n, bits, seed):
    rng = np.random.default_rng(seed)
    keys = rng.integers(0, 1 << bits, n, dtype=np.uint64).astype(np.uint32)
    keys[::5] = keys[0]  # duplicates exercise stability
    vals = rng.permutation(n).astype(np.uint32)
    return np.stack([keys, vals], axis=1)


def test_noalloc_matches_allocating_sort_twice_in_a_row():
    import torch
    assert _abi.lib().brt_radix_sort_noalloc_max_pairs() == 1 << 20
    cases = [(1 << 20, 18, 1), (77777, 12, 2)]  # a large then a smaller call: leftovers must not leak
    for n, bits, seed in cases:
        pairs = _pairs(n, bits, seed)
        din = torch.from_numpy(pairs.view(np.int32)).cuda()
        ref = torch.empty_like(din)
        scratch = torch.empty(radix_sort_scratch_bytes(n, bits), dtype=torch.uint8, device="cuda")
        radix_sort_pairs(din, ref, n, bits, scratch)
        out = torch.full_like(din, -1)
        _noalloc(din, out, n, bits)
        torch.cuda.synchronize()
        got = out.cpu().numpy().view(np.uint32)
        want = ref.cpu().numpy().view(np.uint32)
        assert np.array_equal(got, want), (n, bits)
        order = np.argsort(pairs[:, 0], kind="stable")
        assert np.array_equal(got, pairs[order])


def test_noalloc_leaves_free_device_memory_unchanged():
    """The property the entry point exists for: after one warm-up call (which
    may make the module commit the static array), further calls take no
    device memory."""
    import torch
    n, bits = 300000, 16
    din = torch.from_numpy(_pairs(n, bits, 7).view(np.int32)).cuda()
    out = torch.empty_like(din)
    _noalloc(din, out, n, bits)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(5):
        _noalloc(din, out, n, bits)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0


def test_noalloc_rejects_sizes_beyond_the_static_scratch():
    import torch
    n = (1 << 20) + 1
    din = torch.zeros((n, 2), dtype=torch.int32, device="cuda")
    dout = torch.empty_like(din)
    st = _abi.lib().brt_radix_sort_pairs_noalloc(_abi.ptr(din), _abi.ptr(dout), n, 8, None)
    assert st == _abi.BRT_ERR_CAPACITY
    assert b"1,048,576" in _abi.lib().brt_last_error()
