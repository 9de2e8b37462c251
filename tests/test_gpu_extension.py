"""The plugin extension surface of the C-ABI: registered per-agent arrays move
with their agents through every reorder (single steps, replayed multi-step
graphs, the stage-wise sequence, the autotuner's trials and the adjoint's
recomputation), and work launched with brt_engine_launch runs in stream order
over the engine's own arrays."""
import numpy as np
import pytest
import torch

from behavert_b200 import workloads
from behavert_b200._abi import BrtError, MAX_USER_ARRAYS
from behavert_b200.engine import Engine

pytestmark = pytest.mark.gpu

DT = float(np.float32(0.1))


class _Dev:
    """A device buffer handed to torch through __cuda_array_interface__."""

    def __init__(self, addr, shape, typestr):
        self.__cuda_array_interface__ = {"shape": shape, "typestr": typestr, "data": (int(addr), False),
                                         "strides": None, "version": 2}


def _tensor(addr, shape, typestr="<i4"):
    return torch.as_tensor(_Dev(addr, shape, typestr), device="cuda")


def _engine(n=20000, L=48.0):
    w = workloads.plain(n=n, L=L, M=16, steps=1)
    eng = Engine(w.params)
    eng.set_state(w.pos, w.fwd, w.acc)
    return w, eng


def _device_view(eng, array_id):
    eng.sync()
    v = eng.get_arrays()
    n = v.num_agents
    return (_tensor(v.user[array_id], (n,)).cpu().numpy(), _tensor(v.user_agent_id, (n,)).cpu().numpy(),
            _tensor(v.agent_id, (n,)).cpu().numpy(), _tensor(v.sorted_agent_id, (n,)).cpu().numpy())


def test_arrays_follow_their_agents_through_steps_and_graphs():
    w, eng = _engine()
    with eng:
        n = eng.num_agents
        ids = np.arange(n, dtype=np.uint32)
        tag = eng.add_array(4)
        vec = eng.add_array(16)
        eng.array_set(tag, ids * 7 + 3)
        v = np.random.default_rng(0).random((n, 4)).astype(np.float32)
        eng.array_set(vec, v)
        eng.step(DT, 1)
        eng.step(DT, 5)   # captured once,
        eng.step(DT, 5)   # replayed
        eng.step(DT, 1)
        assert np.array_equal(eng.array_get(tag).ravel(), ids * 7 + 3)
        assert np.array_equal(eng.array_get(vec, np.float32, (n, 4)), v)
        u, uid, aid, _ = _device_view(eng, tag)
        assert np.array_equal(uid, aid)            # the state's slot order
        assert np.array_equal(u, uid * 7 + 3)
        assert not np.array_equal(aid, ids)         # the agents did move


def test_stagewise_reorder_moves_arrays_with_the_sorted_state():
    w, eng = _engine(n=5000, L=32.0)
    with eng:
        n = eng.num_agents
        ids = np.arange(n, dtype=np.uint32)
        tag = eng.add_array(4)
        eng.array_set(tag, ids + 11)
        eng.step(DT, 2)
        eng.reorderSimData()
        u, uid, _, sid = _device_view(eng, tag)
        assert np.array_equal(uid, sid) and np.array_equal(u, sid + 11)
        eng.computeNeighborhoods()
        eng.resetSteerForce()
        eng.computeSeparations()
        eng.computeAlignments()
        eng.computeCohesions()
        eng.computeSeekingsWorldCenter()
        eng.applySteeringForces(DT)
        assert np.array_equal(eng.array_get(tag).ravel(), ids + 11)
        u, uid, aid, _ = _device_view(eng, tag)
        assert np.array_equal(uid, aid)


def test_launch_runs_in_stream_order():
    w, eng = _engine(n=8000, L=40.0)
    with eng:
        n = eng.num_agents
        snap = eng.add_array(16)
        eng.step(DT, 2)
        pos2 = eng.get_state()[0]
        seen = {}

        def work(stream, view):
            seen["n"] = view.num_agents
            with torch.cuda.stream(torch.cuda.ExternalStream(stream)):
                src = _tensor(view.pos4, (view.num_agents, 4), "<f4")
                dst = _tensor(view.user[snap], (view.num_agents, 4), "<f4")
                dst.copy_(src * 2.0)

        eng.launch(work)
        eng.step(DT, 3)
        assert seen["n"] == n
        assert np.array_equal(eng.array_get(snap, np.float32, (n, 4)), pos2 * np.float32(2.0))


def test_launch_reports_the_callbacks_exception():
    w, eng = _engine(n=1000, L=24.0)
    with eng:
        def bad(stream, view):
            raise RuntimeError("from the callback")

        with pytest.raises(RuntimeError, match="from the callback"):
            eng.launch(bad)


def test_autotune_leaves_arrays_with_their_agents():
    w, eng = _engine(n=1 << 15, L=64.0)
    with eng:
        n = eng.num_agents
        ids = np.arange(n, dtype=np.uint32)
        tag = eng.add_array(4)
        eng.array_set(tag, ids * 5 + 1)
        eng.step(DT, 2)
        eng.autotune(DT, steps=2)
        eng.step(DT, 3)
        assert np.array_equal(eng.array_get(tag).ravel(), ids * 5 + 1)
        u, uid, aid, _ = _device_view(eng, tag)
        assert np.array_equal(uid, aid)


def test_adjoint_leaves_arrays_with_their_agents():
    a = workloads.adjoint(n=4096, L=64.0, steps=6)
    with Engine(a.params) as eng:
        eng.set_state(a.pos, a.fwd, a.acc)
        n = eng.num_agents
        ids = np.arange(n, dtype=np.uint32)
        tag = eng.add_array(4)
        eng.array_set(tag, ids * 3 + 2)
        target = np.zeros((n, 4), np.float32)
        target[:, :3] = a.pos[:, :3]
        eng.adjoint_forward(target, 6, 2, a.dt)
        eng.adjoint_backward()
        assert np.array_equal(eng.array_get(tag).ravel(), ids * 3 + 2)
        u, uid, aid, _ = _device_view(eng, tag)
        assert np.array_equal(uid, aid)
        eng.step(a.dt, 2)
        assert np.array_equal(eng.array_get(tag).ravel(), ids * 3 + 2)


def test_bad_registrations_are_rejected():
    w, eng = _engine(n=1000, L=24.0)
    with eng:
        for bad in (0, 6, 2048):
            with pytest.raises(BrtError):
                eng.add_array(bad)
        got = [eng.add_array(8) for _ in range(MAX_USER_ARRAYS)]
        assert got == list(range(MAX_USER_ARRAYS))
        with pytest.raises(BrtError):
            eng.add_array(4)
        with pytest.raises(ValueError):
            eng.array_set(0, np.zeros(eng.num_agents, np.uint32))   # 4 bytes an agent, the array holds 8
