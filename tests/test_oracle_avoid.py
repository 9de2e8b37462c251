"""The oracle's restatement of steerAndSlowToAvoidNeighbors
(OpenSteerWrapper_kernel.cu:110-154) on the CPU: the boosted separation force
and the speed rule, read back through a zero-length step."""
import numpy as np

from behavert_b200 import workloads
from oracle import oracle


def _crowd(ali=0.0, coh=0.0):
    # density 0.064 a unit^3: about 17 agents within the radius, so both
    # branches of the neighbour-count boost occur
    w = workloads.plain(n=4096, L=40.0, M=32, seed=5, steps=1)
    w.params[0].alignmentParams[0] = ali
    w.params[0].cohesionParams[0] = coh
    return w


def test_force_boost_and_speed_rule():
    w = _crowd()
    f64 = [a.astype(np.float64) for a in (w.pos, w.fwd, w.acc)]
    o = oracle.step(w.params, *f64, dt=0.0, mode=1, avoid_neighbors=True)
    ids = o["ids"]
    n = o["lists"][:, 0].astype(np.int64)
    steer = o["steer"][:, :3]                      # per sorted slot
    fin = f64[1][ids]                              # input forward per sorted slot
    mag = np.linalg.norm(steer, axis=1)
    boost = np.where(n > 16, (n - 16) * 0.5, 1.0)
    some = mag > 0
    assert some.mean() > 0.9
    assert np.allclose(mag[some], 1.5 * boost[some], rtol=1e-9)
    assert (n > 16).sum() > 100 and (n <= 16).sum() > 100
    d = np.sum(steer * fin[:, :3], axis=1)
    factor = np.where(d < -0.8, 0.9, np.where(d > 0.5, 1.02, 1.0))
    assert (factor == 0.9).sum() > 50 and (factor == 1.02).sum() > 50 and (factor == 1.0).sum() > 50
    # dt = 0: the integration keeps the position and returns |forward * speed|
    # capped at maxSpeed 1
    speed = fin[:, 3] * factor * np.linalg.norm(fin[:, :3], axis=1)
    assert np.allclose(o["fwd"][ids, 3], np.minimum(speed, 1.0), rtol=1e-9, atol=1e-12)
    assert np.array_equal(o["pos"][:, :3], f64[0][:, :3])


def test_crowd_order_differs_from_flocking_order_only_by_the_stage():
    w = _crowd(ali=1.0, coh=1.0)
    a = oracle.step(w.params, w.pos, w.fwd, w.acc, dt=w.dt, mode=0, avoid_neighbors=True)
    b = oracle.step(w.params, w.pos, w.fwd, w.acc, dt=w.dt, mode=0, avoid_neighbors=False)
    assert np.array_equal(a["lists"], b["lists"])
    assert not np.array_equal(a["fwd"], b["fwd"])
    # the force is the same in both orders where the boost is 1 (at most 16
    # neighbours, or exactly 18) and differs where it is 0.5 or above 1; the
    # speed rule does not feed back into these stages' forces
    n = a["lists"][:, 0]
    same = np.all(a["steer"] == b["steer"], axis=1)
    one = (n <= 16) | (n == 18)
    assert same[one].all()
    assert not same[~one].any()


def test_fp32_close_to_fp64():
    w = _crowd(ali=1.0, coh=1.0)
    a = oracle.step(w.params, w.pos, w.fwd, w.acc, dt=w.dt, mode=0, avoid_neighbors=True)
    f64 = [x.astype(np.float64) for x in (w.pos, w.fwd, w.acc)]
    b = oracle.step(w.params, *f64, dt=w.dt, mode=1, avoid_neighbors=True)
    assert np.array_equal(a["lists"], b["lists"])
    assert np.max(np.abs(oracle.min_image(a["pos"][:, :3] - b["pos"][:, :3], 40.0))) < 1e-5
    va = a["fwd"][:, :3] * a["fwd"][:, 3:4]
    vb = b["fwd"][:, :3] * b["fwd"][:, 3:4]
    assert np.linalg.norm(va - vb) / np.linalg.norm(vb) < 1e-5


def test_move_away_from_base_force():
    """steerForMoveAwayBaseTarget alone: (w * (p - base)) / |p - base| within
    twice the radius, zero beyond (OpenSteerWrapper_kernel.cu:185-212)."""
    w = _crowd()
    w.params[0].separationParams[0] = 0.0
    base, prm = (20.0, 15.0, 25.0), (2.0, 500.0, 8.0)
    f64 = [a.astype(np.float64) for a in (w.pos, w.fwd, w.acc)]
    o = oracle.step(w.params, *f64, dt=0.1, mode=1, move_away=(base, prm))
    p = f64[0][o["ids"], :3]
    off = p - np.array(base)
    d = np.linalg.norm(off, axis=1)
    expect = np.where((d > 2 * prm[2])[:, None], 0.0, prm[0] * off / d[:, None])
    assert (d <= 2 * prm[2]).sum() > 100 and (d > 2 * prm[2]).sum() > 100
    assert np.allclose(o["steer"][:, :3], expect, rtol=1e-12, atol=1e-12)
    plain = oracle.step(w.params, *f64, dt=0.1, mode=1)
    assert np.all(plain["steer"][:, :3] == 0.0)
