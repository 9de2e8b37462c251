"""The FP64 frozen-neighbour / frozen-branch model of the oracle
(oracle/brt_oracle_adjoint.cpp): its forward against the oracle's own FP64
step, and its hand-written reverse mode against central finite differences.
CPU only; this pins the reference the CUDA adjoint is checked against."""
import copy

import numpy as np
import pytest

from behavert_b200 import workloads
from oracle import oracle

T_STEPS = 8


def _params_with(params, w):
    out = []
    for p in params:
        q = copy.copy(p)
        q.separationParams[0], q.alignmentParams[0], q.cohesionParams[0] = (float(x) for x in w)
        out.append(q)
    return out


def _velocity_to_state(v):
    s = np.linalg.norm(v, axis=1)
    fwd = np.zeros((len(v), 4))
    fwd[:, :3] = v / s[:, None]
    fwd[:, 3] = s
    return fwd


def _slow_obstacles(wl):
    """Speeds around the low-speed limit (0.2 maxSpeed) so that
    adjustRawSteeringForce limits the deviation, a high maxForce share of
    clipped forces, and static sphere obstacles."""
    rng = np.random.default_rng(21)
    p = wl.params[0]
    p.numObstacles = 8
    p.obstacleAvoidanceWeight = 2.0
    for o in range(8):
        c = rng.uniform(0, p.worldSize, 3)
        p.obstacles[o][0], p.obstacles[o][1], p.obstacles[o][2] = (float(x) for x in c)
        p.obstacles[o][3] = float(rng.uniform(2, 5))
    wl.fwd[:, 3] = rng.uniform(0.05, 0.3, len(wl.fwd)).astype(np.float32)
    return wl


@pytest.fixture(scope="module", params=["plain", "slow_obstacles"])
def problem(request):
    wl = workloads.adjoint(n=2048, L=32.0, steps=T_STEPS)
    if request.param == "slow_obstacles":
        wl = _slow_obstacles(wl)
    params = wl.params
    L = float(params[0].worldSize)
    pos = wl.pos.astype(np.float64)
    fwd = wl.fwd.astype(np.float64)
    acc = wl.acc.astype(np.float64)
    # FP64 oracle steps give the per-step neighbour lists and the trajectory.
    lists, p_, f_, a_ = [], pos, fwd, acc
    for _ in range(T_STEPS):
        out = oracle.step(params, p_, f_, a_, dt=wl.dt, mode=1)
        lists.append(oracle.lists_by_id(out))
        p_, f_, a_ = out["pos"], out["fwd"], out["acc"]
    lists = np.stack(lists)
    rng = np.random.default_rng(11)
    target = p_[:, :3] + rng.normal(0.0, 0.5, (len(p_), 3))
    # The oracle's step (like the CUDA library) takes dt as a float.
    dt = float(np.float32(wl.dt))
    return dict(wl=wl, params=params, L=L, pos=pos, fwd=fwd, acc=acc, lists=lists, final=(p_, f_, a_), target=target,
                dt=dt)


def _loss(pr, out):
    d = oracle.min_image(out["pos"][:, :3] - pr["target"], pr["L"])
    return float(np.mean(np.sum(d * d, axis=1)))


def test_frozen_forward_matches_oracle_fp64_steps(problem):
    pr = problem
    out = oracle.frozen_forward(pr["params"], pr["pos"], pr["fwd"], pr["acc"], pr["lists"], dt=pr["dt"])
    p_, f_, a_ = pr["final"]
    dp = oracle.min_image(out["pos"][:, :3] - p_[:, :3], pr["L"])
    assert np.max(np.abs(dp)) < 1e-9
    assert np.max(np.abs(out["fwd"] - f_)) < 1e-9
    assert np.max(np.abs(out["acc"][:, :3] - a_[:, :3])) < 1e-9


def test_frozen_flags_reproduce_trajectory(problem):
    pr = problem
    base = oracle.frozen_forward(pr["params"], pr["pos"], pr["fwd"], pr["acc"], pr["lists"], dt=pr["dt"],
                                 want_flags=True)
    again = oracle.frozen_forward(pr["params"], pr["pos"], pr["fwd"], pr["acc"], pr["lists"], dt=pr["dt"],
                                  flags=base["flags"])
    for k in ("pos", "fwd", "acc"):
        assert np.array_equal(base[k], again[k])
    f = base["flags"]
    assert np.any(f[..., 1] != 0) and np.any(f[..., 2] != 0) and np.any(f[..., 3] != 0)
    if pr["params"][0].numObstacles:
        assert np.any(f[..., 0] & 3 == 3)  # low-speed deviation limit taken
        assert np.any(f[..., 0] & 4)       # steering force clipped to maxForce
    else:
        assert np.any(f[..., 0] & 8)       # velocities clipped to maxSpeed


def test_reverse_matches_central_differences(problem):
    pr = problem
    params, dt = pr["params"], pr["dt"]
    w0 = np.array([[params[0].separationParams[0], params[0].alignmentParams[0], params[0].cohesionParams[0]]])
    base = oracle.frozen_forward(params, pr["pos"], pr["fwd"], pr["acc"], pr["lists"], weights=w0, dt=dt,
                                 want_flags=True)
    flags = base["flags"]
    n = len(pr["pos"])
    gpos_T = np.zeros((n, 4))
    gpos_T[:, :3] = 2.0 / n * oracle.min_image(base["pos"][:, :3] - pr["target"], pr["L"])
    rev = oracle.frozen_reverse(params, pr["pos"], pr["fwd"], pr["acc"], pr["lists"], gpos_T, weights=w0,
                                flags=flags, dt=dt)
    f0, s0 = pr["fwd"][:, :3], pr["fwd"][:, 3]
    gf, gs = rev["fwd"][:, :3], rev["fwd"][:, 3]
    gvel = gs[:, None] * f0 + (gf - f0 * np.sum(f0 * gf, axis=1)[:, None]) / s0[:, None]

    def loss_at(w=w0, pos=pr["pos"], fwd=pr["fwd"]):
        out = oracle.frozen_forward(params, pos, fwd, pr["acc"], pr["lists"], weights=w, flags=flags, dt=dt)
        return _loss(pr, out)

    # Richardson-extrapolated central differences: pow(speed / limit, 20) in
    # the low-speed branch makes the plain O(h^2) error visible at 1e-6.
    h = 1e-5

    def fd(fn):
        d1 = (fn(h) - fn(-h)) / (2 * h)
        d2 = (fn(h / 2) - fn(-h / 2)) / h
        return (4 * d2 - d1) / 3

    def close(a, b):
        return abs(a - b) <= 1e-6 * max(abs(a), abs(b)) + 1e-10

    for b in range(3):
        def fw(e, b=b):
            w = w0.copy()
            w[0, b] += e
            return loss_at(w=w)
        d = fd(fw)
        assert close(d, rev["weights"][0, b]), ("w", b, d, rev["weights"][0, b])
    rng = np.random.default_rng(5)
    agents = rng.choice(n, 6, replace=False)
    v0 = f0 * s0[:, None]
    for i in agents:
        for c in range(3):
            def fp(e, i=i, c=c):
                p = pr["pos"].copy()
                p[i, c] += e
                return loss_at(pos=p)

            def fv(e, i=i, c=c):
                v = v0[i:i + 1].copy()
                v[0, c] += e
                f = pr["fwd"].copy()
                f[i] = _velocity_to_state(v)[0]
                return loss_at(fwd=f)
            d = fd(fp)
            assert close(d, rev["pos"][i, c]), ("pos", i, c, d, rev["pos"][i, c])
            d = fd(fv)
            assert close(d, gvel[i, c]), ("vel", i, c, d, gvel[i, c])
