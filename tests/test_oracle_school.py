"""The oracle's restatement of the Schooling law (CPU): constant speed,
unit headings, the turn limit, and FP32 against FP64."""
import numpy as np
import pytest

from behavert_b200 import workloads
from oracle import oracle


@pytest.mark.parametrize("mode", [1, 2])
def test_constant_speed_and_turn_limit(mode):
    w = workloads.schooling(n=2048, L=32.0, mode=mode)
    o = oracle.step(w.params, w.pos, w.fwd, w.acc, dt=w.dt, mode=1, random_step=1)
    p = w.params[0].schooling
    step = 0.1 if mode == 1 else 0.2
    d = oracle.min_image(o["pos"][:, :3] - w.pos[:, :3], 32.0)
    assert np.allclose(np.linalg.norm(d, axis=1), p.s * step, rtol=1e-5)
    assert np.allclose(np.linalg.norm(o["fwd"][:, :3], axis=1), 1.0, atol=1e-5)
    assert np.all(o["fwd"][:, 3] == np.float32(p.s))
    cos = np.sum(o["fwd"][:, :3] * w.fwd[:, :3], axis=1)
    assert np.all(cos >= p.theta - 1e-5)


@pytest.mark.parametrize("mode", [1, 2])
def test_fp32_close_to_fp64(mode):
    w = workloads.schooling(n=2048, L=32.0, mode=mode)
    a = oracle.step(w.params, w.pos, w.fwd, w.acc, dt=w.dt, mode=0, random_step=3)
    b = oracle.step(w.params, w.pos, w.fwd, w.acc, dt=w.dt, mode=1, random_step=3)
    assert np.array_equal(a["lists"], b["lists"])
    assert np.max(np.abs(oracle.min_image(a["pos"][:, :3] - b["pos"][:, :3], 32.0))) < 1e-4
    assert np.max(np.abs(a["fwd"] - b["fwd"])) < 1e-3


def test_random_stream_depends_on_step_and_seed():
    w = workloads.schooling(n=1024, L=32.0, mode=2, random_weight=0.5)
    a = oracle.step(w.params, w.pos, w.fwd, w.acc, mode=0, random_step=1)
    b = oracle.step(w.params, w.pos, w.fwd, w.acc, mode=0, random_step=1)
    c = oracle.step(w.params, w.pos, w.fwd, w.acc, mode=0, random_step=2)
    assert np.array_equal(a["fwd"], b["fwd"])
    assert not np.array_equal(a["fwd"], c["fwd"])
