"""The autotuner and the launch options it chooses between: every option
leaves the results bit-identical, and autotuning leaves the state alone."""
import numpy as np
import pytest

from behavert_b200 import workloads
from behavert_b200.engine import Engine

pytestmark = pytest.mark.gpu

DT = float(np.float32(0.1))


def _run(wl, steps, options=()):
    with Engine(wl.params) as eng:
        for k, v in options:
            eng.set_option(k, v)
        eng.set_state(wl.pos, wl.fwd, wl.acc, wl.feat)
        eng.step(DT, steps)
        return eng.get_state()


@pytest.mark.parametrize("block", [32, 64, 96, 256])
def test_block_sizes_are_bit_identical(block):
    wl = workloads.large(n=1 << 15, steps=3)
    ref = _run(wl, 3)
    out = _run(wl, 3, [("block_size", block)])
    for a, b in zip(ref, out):
        assert np.array_equal(a, b)


def _variant_workloads():
    big = workloads.large(n=1 << 15, steps=2)
    bat = workloads.batched(num_flocks=12, lo=128, hi=6000, steps=2)
    cap = workloads.plain(n=4096, L=32.0, steps=2)
    cap.params[0].maxBodiesPerCell = 3
    seam = workloads.plain(n=1500, L=12.0, M=32, steps=2)   # 3 cells per side: every cell is on a seam
    flat = workloads.plain(n=3000, L=32.0, steps=2)
    flat.params[0].use2DProjection = 1
    odd = workloads.plain(n=1000, L=32.0, steps=2)          # not a multiple of the warp size
    # dense rows: the staged tile kernel's neighbourhood overflows its shared
    # memory in some tiles and not in others
    dense = workloads.large(n=1 << 15, L=48.0, blobs=3, blob_fraction=0.6, steps=2)
    return {"large": big, "batched": bat, "cap": cap, "seam": seam, "2d": flat, "odd": odd, "dense": dense}


@pytest.mark.parametrize("variant", [1, 2, 3, 4, 5, 6, 7])
@pytest.mark.parametrize("name", ["large", "batched", "cap", "seam", "2d", "odd", "dense"])
def test_scan_variants_are_bit_identical(name, variant):
    wl = _variant_workloads()[name]

    def run(options):
        with Engine(wl.params) as eng:
            for k, v in options:
                eng.set_option(k, v)
            eng.record_lists(True)
            eng.set_state(wl.pos, wl.fwd, wl.acc, wl.feat)
            eng.step(DT, 2)
            return eng.getNeighborLists(), eng.get_state()

    ref_lists, ref = run([])
    lists, out = run([("scan_variant", variant)])
    assert np.array_equal(lists[:, 0], ref_lists[:, 0])
    for i in range(len(lists)):
        n = lists[i, 0]
        assert np.array_equal(lists[i, 1:1 + n], ref_lists[i, 1:1 + n]), i
    for a, b in zip(ref, out):
        if a is not None:
            assert np.array_equal(a, b)


@pytest.mark.parametrize("scan,phase2", [(0, 1), (4, 2), (4, 1), (5, 2), (6, 2), (7, 2), (7, 0)])
@pytest.mark.parametrize("name", ["large", "batched", "seam"])
def test_list_walk_variants_are_bit_identical(name, scan, phase2):
    wl = _variant_workloads()[name]
    ref = _run(wl, 2, [("scan_variant", scan)])
    for regs in (64, 48):
        out = _run(wl, 2, [("scan_variant", scan), ("phase2_variant", phase2), ("registers", regs)])
        for a, b in zip(ref, out):
            if a is not None:
                assert np.array_equal(a, b)


@pytest.mark.parametrize("scan", [4, 7])
@pytest.mark.parametrize("budget", [128, 48, 40])
@pytest.mark.parametrize("name", ["large", "batched", "seam"])
def test_register_budgets_are_bit_identical(name, budget, scan):
    wl = _variant_workloads()[name]
    ref = _run(wl, 2, [("scan_variant", scan)])
    out = _run(wl, 2, [("scan_variant", scan), ("registers", budget)])
    for a, b in zip(ref, out):
        if a is not None:
            assert np.array_equal(a, b)


def test_bad_register_budget_is_rejected():
    from behavert_b200._abi import BrtError
    wl = workloads.plain(n=512, L=32.0, steps=1)
    with Engine(wl.params) as eng:
        for bad in (0, 32, 96, 256):
            with pytest.raises(BrtError):
                eng.set_option("registers", bad)


def test_sort_digit_widths_cap_at_four_passes():
    # 18-bit keys with 4-bit digits would need 5 passes; the plan widens them.
    wl = workloads.large(n=1 << 15, L=256.0, steps=2)
    ref = _run(wl, 2)
    for bits in (4, 5, 9):
        out = _run(wl, 2, [("sort_digit_bits", bits)])
        for a, b in zip(ref, out):
            assert np.array_equal(a, b)


def test_bad_block_size_is_rejected():
    from behavert_b200._abi import BrtError
    wl = workloads.plain(n=512, L=32.0, steps=1)
    with Engine(wl.params) as eng:
        for bad in (0, 48, 512):
            with pytest.raises(BrtError):
                eng.set_option("block_size", bad)


def test_autotune_keeps_state_and_results():
    wl = workloads.large(n=1 << 16, steps=4)
    ref = _run(wl, 4)
    with Engine(wl.params) as eng:
        eng.set_state(wl.pos, wl.fwd, wl.acc, wl.feat)
        before = eng.get_state()
        rep = eng.autotune(DT, steps=3)
        after = eng.get_state()
        for a, b in zip(before, after):
            assert np.array_equal(a, b)
        assert 4 <= rep["sort_digit_bits"] <= 9 and rep["block_size"] in (64, 128, 256)
        assert len(rep["trials"]) >= 5 and rep["ms_per_step"] > 0
        eng.step(DT, 4)
        out = eng.get_state()
    for a, b in zip(ref, out):
        assert np.array_equal(a, b)


def test_engines_with_different_list_lengths_coexist():
    """Kernel shared-memory limits are per device: an engine created later
    with short lists must not lower the limit an earlier engine with long
    lists needs (here 257 x 100 list words a block, above the default 48 KB)."""
    big = workloads.plain(n=4096, L=32.0, M=100, steps=1)
    small = workloads.plain(n=2048, L=32.0, M=8, steps=1)
    ref = _run(big, 2, [("block_size", 256)])
    with Engine(big.params) as a:
        a.set_option("block_size", 256)
        a.set_state(big.pos, big.fwd, big.acc, big.feat)
        a.step(DT, 1)
        with Engine(small.params) as b:
            b.set_state(small.pos, small.fwd, small.acc, small.feat)
            b.step(DT, 1)
            a.step(DT, 1)
            out = a.get_state()
    for x, y in zip(ref, out):
        if x is not None:
            assert np.array_equal(x, y)
