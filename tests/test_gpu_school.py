"""The Schooling law on the GPU (fused step and the reference's stage-wise
functionalities) against the FP32 oracle: neighbour lists, sorted order and
state bit-exact (the law uses only + - * / and sqrt, correctly rounded on
both sides), and against the FP64 oracle within 1e-4."""
import numpy as np
import pytest

from behavert_b200 import workloads
from behavert_b200.engine import Engine
from behavert_b200._abi import BrtError, lib, check

pytestmark = pytest.mark.gpu


def _oracle():
    from oracle import oracle
    return oracle


def _gpu_steps(w, steps, record=False):
    with Engine(w.params) as eng:
        eng.record_lists(record)
        eng.set_state(w.pos, w.fwd, w.acc)
        eng.step(w.dt, steps)
        out = eng.get_state(features=False)
        extra = (eng.getHash(), eng.getNeighborLists()) if record else None
    return out, extra


@pytest.mark.parametrize("mode", [1, 2])
def test_one_step_bit_exact(mode):
    o = _oracle()
    w = workloads.schooling(n=4096, L=64.0, mode=mode)
    (pos, fwd, acc, _), ((keys, ids), lists) = _gpu_steps(w, 1, record=True)
    r = o.step(w.params, w.pos, w.fwd, w.acc, dt=w.dt, mode=0, random_step=1)
    assert np.array_equal(keys, r["keys"]) and np.array_equal(ids, r["ids"])
    assert np.array_equal(lists[:, 0], r["lists"][:, 0])
    for i in range(len(lists)):
        n = lists[i, 0]
        assert np.array_equal(lists[i, 1:1 + n], r["lists"][i, 1:1 + n])
    assert np.array_equal(pos, r["pos"])
    assert np.array_equal(fwd, r["fwd"])
    assert np.array_equal(acc, r["acc"])
    r64 = o.step(w.params, w.pos, w.fwd, w.acc, dt=w.dt, mode=1, random_step=1)
    d = o.min_image(pos[:, :3].astype(np.float64) - r64["pos"][:, :3], 64.0)
    assert np.max(np.abs(d)) < 1e-4


@pytest.mark.parametrize("mode", [1, 2])
def test_non_finite_and_outside_positions(mode):
    """NaN agents (every axis, one axis) beside finite agents in cell 0,
    infinite coordinates and agents outside the world: lists, order and state
    as the oracle's, NaN for NaN."""
    from tests.test_gpu_parity import _same_bits
    o = _oracle()
    w = workloads.schooling(n=600, L=16.0, mode=mode)
    rng = np.random.default_rng(7)
    w.pos[:40, :3] = (rng.random((40, 3)) * 3.0).astype(np.float32)
    w.pos[40:43, :3] = np.nan
    w.pos[43, 0] = np.nan
    w.pos[44, 1] = np.inf
    w.pos[45, 2] = -np.inf
    w.pos[46, 0] = -3.0
    w.pos[47, 0] = 21.0
    (pos, fwd, acc, _), ((keys, ids), lists) = _gpu_steps(w, 1, record=True)
    r = o.step(w.params, w.pos, w.fwd, w.acc, dt=w.dt, mode=0, random_step=1)
    assert np.array_equal(keys, r["keys"]) and np.array_equal(ids, r["ids"])
    cnt = lists[:, 0]
    assert np.array_equal(cnt, r["lists"][:, 0])
    mask = np.arange(lists.shape[1] - 1)[None, :] < cnt[:, None]
    assert np.array_equal(np.where(mask, lists[:, 1:], 0), np.where(mask, r["lists"][:, 1:], 0))
    assert _same_bits(pos, r["pos"]) and _same_bits(fwd, r["fwd"]) and _same_bits(acc, r["acc"])


@pytest.mark.parametrize("mode", [1, 2])
def test_full_size_two_steps_bit_exact(mode):
    """1,048,576 agents in the cube of side 256 (the size the benchmark
    measures): two steps, lists, order and state bit-exact."""
    o = _oracle()
    w = workloads.schooling(n=1 << 20, L=256.0, mode=mode)
    with Engine(w.params) as eng:
        eng.set_state(w.pos, w.fwd, w.acc)
        p, f, a = w.pos, w.fwd, w.acc
        for s in range(2):
            eng.record_lists(True)
            eng.step(w.dt, 1)
            keys, ids = eng.getHash()
            lists = eng.getNeighborLists()
            pos, fwd, acc, _ = eng.get_state(features=False)
            r = o.step(w.params, p, f, a, dt=w.dt, mode=0, random_step=s + 1)
            assert np.array_equal(keys, r["keys"]) and np.array_equal(ids, r["ids"])
            cnt = lists[:, 0]
            assert np.array_equal(cnt, r["lists"][:, 0])
            mask = np.arange(lists.shape[1] - 1)[None, :] < cnt[:, None]
            assert np.array_equal(np.where(mask, lists[:, 1:], 0), np.where(mask, r["lists"][:, 1:], 0))
            assert np.array_equal(pos, r["pos"]) and np.array_equal(fwd, r["fwd"]) and np.array_equal(acc, r["acc"])
            p, f, a = pos, fwd, acc


@pytest.mark.parametrize("mode", [1, 2])
def test_ten_steps_bit_exact(mode):
    o = _oracle()
    w = workloads.schooling(n=4096, L=64.0, mode=mode)
    (pos, fwd, acc, _), _ = _gpu_steps(w, 10)
    p, f, a = w.pos, w.fwd, w.acc
    for s in range(10):
        r = o.step(w.params, p, f, a, dt=w.dt, mode=0, random_step=s + 1, want_intermediates=False)
        p, f, a = r["pos"], r["fwd"], r["acc"]
    assert np.array_equal(pos, p) and np.array_equal(fwd, f)


def test_stagewise_equals_fused_split_path():
    w = workloads.schooling(n=4096, L=64.0, mode=2)
    (pos, fwd, acc, _), _ = _gpu_steps(w, 1)
    o = _oracle()
    r = o.step(w.params, w.pos, w.fwd, w.acc, dt=w.dt, mode=0, random_step=1)
    with Engine(w.params) as eng:
        eng.set_state(w.pos, w.fwd, w.acc)
        eng.reorderSimData()
        eng.computeNeighborhoods()
        check(lib().brt_school_repulsion(eng.handle), "repulsion")
        check(lib().brt_school_attraction_orientation(eng.handle), "attraction/orientation")
        steer = eng.getSteerForce()
        check(lib().brt_school_movement(eng.handle), "movement")
        s_pos, s_fwd, s_acc, _ = eng.get_state(features=False)
    assert np.array_equal(steer, r["steer"])
    assert np.array_equal(s_pos, pos) and np.array_equal(s_fwd, fwd) and np.array_equal(s_acc, acc)


def test_stagewise_equals_fused_animate():
    w = workloads.schooling(n=4096, L=64.0, mode=1)
    (pos, fwd, _, _), _ = _gpu_steps(w, 1)
    with Engine(w.params) as eng:
        eng.set_state(w.pos, w.fwd, w.acc)
        eng.reorderSimData()
        eng.computeNeighborhoods()
        check(lib().brt_school_animate(eng.handle), "animateSchool")
        s_pos, s_fwd, _, _ = eng.get_state(features=False)
    assert np.array_equal(s_pos, pos) and np.array_equal(s_fwd, fwd)


def test_batched_schools_and_random_step_option():
    o = _oracle()
    w = workloads.schooling(n=1500, L=48.0, mode=2, flocks=3, random_weight=0.3)
    with Engine(w.params) as eng:
        eng.set_option("random_step", 41)
        eng.set_state(w.pos, w.fwd, w.acc)
        eng.step(w.dt, 1)
        pos, fwd, _, _ = eng.get_state(features=False)
    r = o.step(w.params, w.pos, w.fwd, w.acc, dt=w.dt, mode=0, random_step=42, want_intermediates=False)
    assert np.array_equal(pos, r["pos"]) and np.array_equal(fwd, r["fwd"])


def test_mixed_families_are_rejected():
    a = workloads.schooling(n=512, L=32.0, mode=1)
    b = workloads.plain(n=512, L=32.0, steps=1)
    with pytest.raises(BrtError):
        Engine([a.params[0], b.params[0]])
    with Engine(b.params) as eng:
        eng.set_state(b.pos, b.fwd, b.acc)
        eng.reorderSimData()
        eng.computeNeighborhoods()
        assert lib().brt_school_animate(eng.handle) != 0
