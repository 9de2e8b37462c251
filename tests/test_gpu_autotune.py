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
