"""The incremental re-sort: a fused step whose order comes from the previous
step's must equal the full radix sort's, whichever way the device decides
(few movers, many movers, a crowded cell, a replaced state, a stage-wise
step in between)."""
import numpy as np
import pytest

from behavert_b200 import workloads
from behavert_b200.engine import Engine

pytestmark = pytest.mark.gpu

DT = float(np.float32(0.1))


def _workloads():
    big = workloads.large(n=1 << 15, steps=2)
    bat = workloads.batched(num_flocks=12, lo=128, hi=6000, steps=2)
    cap = workloads.plain(n=4096, L=32.0, steps=2)
    cap.params[0].maxBodiesPerCell = 3
    seam = workloads.plain(n=1500, L=12.0, M=32, steps=2)
    flat = workloads.plain(n=3000, L=32.0, steps=2)
    flat.params[0].use2DProjection = 1
    odd = workloads.plain(n=1000, L=32.0, steps=2)
    return {"large": big, "batched": bat, "cap": cap, "seam": seam, "2d": flat, "odd": odd}


def _trajectory(wl, incremental, chunks, dt=DT):
    """State, sorted order and cell ranges after each chunk of steps (a
    chunk of 1 is a single launch, more a graph)."""
    out = []
    with Engine(wl.params) as eng:
        eng.set_option("incremental_sort", int(incremental))
        eng.set_state(wl.pos, wl.fwd, wl.acc, wl.feat)
        for k in chunks:
            eng.step(dt, k)
            out.append((eng.get_state(), eng.getHash(), eng.getCellRanges()))
        assert eng.device_error() == 0
    return out


def _same(a, b):
    for (sa, ha, ca), (sb, hb, cb) in zip(a, b):
        for x, y in zip(sa, sb):
            if x is not None:
                assert np.array_equal(x.view(np.uint32), y.view(np.uint32))
        for x, y in zip(ha, hb):
            assert np.array_equal(x, y)
        for x, y in zip(ca, cb):
            assert np.array_equal(x, y)


@pytest.mark.parametrize("name", ["large", "batched", "cap", "seam", "2d", "odd"])
def test_incremental_equals_full_sort(name):
    wl = _workloads()[name]
    chunks = [1, 1, 1, 5, 1, 12]
    _same(_trajectory(wl, True, chunks), _trajectory(wl, False, chunks))


def test_many_movers_fall_back_to_the_full_sort():
    # a long step moves far more than one agent in eight to another cell
    wl = workloads.plain(n=4096, L=32.0, steps=2)
    chunks = [1, 1, 3]
    _same(_trajectory(wl, True, chunks, dt=8.0), _trajectory(wl, False, chunks, dt=8.0))


def test_crowded_cell_falls_back_to_the_full_sort():
    # 48 agents just below a cell face, all heading across it together: one
    # cell receives more movers than its list holds (headings differ a little:
    # identical ones make the alignment term normalise a zero vector)
    wl = workloads.plain(n=2048, L=32.0, steps=2)
    pos, fwd = wl.pos.copy(), wl.fwd.copy()
    k = 48
    rng = np.random.default_rng(7)
    pos[:k, 0] = 15.98
    pos[:k, 1] = 17.0 + rng.random(k, dtype=np.float32) * 2.0
    pos[:k, 2] = 9.0 + rng.random(k, dtype=np.float32) * 2.0
    head = np.stack([np.ones(k), 0.05 * rng.standard_normal(k), 0.05 * rng.standard_normal(k)], axis=1)
    fwd[:k, :3] = (head / np.linalg.norm(head, axis=1, keepdims=True)).astype(np.float32)
    fwd[:k, 3] = 1.0
    wl.pos, wl.fwd = pos, fwd
    chunks = [1, 1, 1, 4]
    _same(_trajectory(wl, True, chunks), _trajectory(wl, False, chunks))


def test_replaced_state_takes_the_full_sort():
    a = workloads.plain(n=4096, L=32.0, steps=2, seed=0)
    b = workloads.plain(n=4096, L=32.0, steps=2, seed=5)
    with Engine(a.params) as eng, Engine(b.params) as ref:
        eng.set_state(a.pos, a.fwd, a.acc, a.feat)
        eng.step(DT, 4)
        eng.set_state(b.pos, b.fwd, b.acc, b.feat)
        eng.step(DT, 1)
        eng.step(DT, 6)
        ref.set_option("incremental_sort", 0)
        ref.set_state(b.pos, b.fwd, b.acc, b.feat)
        ref.step(DT, 1)
        ref.step(DT, 6)
        for x, y in zip(eng.get_state(), ref.get_state()):
            if x is not None:
                assert np.array_equal(x, y)
        for x, y in zip(eng.getHash(), ref.getHash()):
            assert np.array_equal(x, y)


def test_stagewise_step_between_fused_steps():
    wl = workloads.large(n=20000)
    with Engine(wl.params) as a, Engine(wl.params) as b:
        b.set_option("incremental_sort", 0)
        for eng in (a, b):
            eng.set_state(wl.pos, wl.fwd, wl.acc, wl.feat)
            eng.step(DT, 3)
            eng.update_stagewise(DT)
            eng.step(DT, 1)
            eng.step(DT, 3)
        for x, y in zip(a.get_state(), b.get_state()):
            if x is not None:
                assert np.array_equal(x, y)
        cs_a, ce_a = a.getCellRanges()
        cs_b, ce_b = b.getCellRanges()
        assert np.array_equal(cs_a, cs_b) and np.array_equal(ce_a, ce_b)
