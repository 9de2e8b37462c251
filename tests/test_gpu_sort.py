"""GPU tests of the standalone onesweep sort (brt_radix_sort_pairs) against a
stable numpy sort, and of the sort inside the engine on adversarial keys."""
import numpy as np
import pytest

from behavert_b200 import radix_sort_pairs, radix_sort_scratch_bytes

pytestmark = pytest.mark.gpu


def _sort_gpu(keys, vals, bits):
    import torch
    n = len(keys)
    pairs = np.stack([keys, vals], axis=1).astype(np.uint32)
    din = torch.from_numpy(pairs.view(np.int32)).cuda()
    dout = torch.empty_like(din)
    scratch = torch.empty(radix_sort_scratch_bytes(n, bits), dtype=torch.uint8, device="cuda")
    radix_sort_pairs(din, dout, n, bits, scratch)
    torch.cuda.synchronize()
    return dout.cpu().numpy().view(np.uint32)


@pytest.mark.parametrize("n,bits", [(1, 8), (7, 4), (2047, 12), (2048, 12), (2049, 18), (100000, 18),
                                    (1 << 20, 18), (300001, 24), (65536, 32), (5000, 1)])
def test_sort_matches_stable_numpy(n, bits):
    rng = np.random.default_rng(n + bits)
    hi = (1 << bits) if bits < 32 else (1 << 32)
    keys = rng.integers(0, hi, n, dtype=np.uint64).astype(np.uint32)
    vals = np.arange(n, dtype=np.uint32)
    out = _sort_gpu(keys, vals, bits)
    order = np.argsort(keys, kind="stable")
    assert np.array_equal(out[:, 0], keys[order])
    assert np.array_equal(out[:, 1], vals[order])


def test_sort_low_bits_only_and_duplicates():
    rng = np.random.default_rng(5)
    n = 50000
    keys = rng.integers(0, 1 << 30, n, dtype=np.uint64).astype(np.uint32)
    keys[::3] = 7  # heavy duplicates
    vals = rng.permutation(n).astype(np.uint32)
    out = _sort_gpu(keys, vals, 10)
    low = keys & 1023
    order = np.argsort(low, kind="stable")
    assert np.array_equal(out[:, 1], vals[order])
    assert np.array_equal(out[:, 0], keys[order])


def test_sort_all_equal_and_presorted():
    n = 70000
    keys = np.zeros(n, np.uint32)
    vals = np.arange(n, dtype=np.uint32)
    out = _sort_gpu(keys, vals, 16)
    assert np.array_equal(out[:, 1], vals)
    keys = np.arange(n, dtype=np.uint32)
    out = _sort_gpu(keys[::-1].copy(), vals, 17)
    assert np.array_equal(out[:, 0], keys)
