"""The CUDA adjoint (brt_adjoint_forward / brt_adjoint_backward) against the
FP64 frozen-neighbour, frozen-branch oracle fed with the GPU's own frozen
lists and branch decisions, and against FP64 central finite differences.

Tolerances: the gradient is of the FP32 forward; the FP64 reference runs
the same frozen model in double precision, so differences come from FP32
rounding of the trajectory and of the adjoint arithmetic.  Weight gradients
and sampled state coordinates must match to 1e-4 relative (the coordinate
check has an absolute floor of 1e-4 of the median gradient magnitude)."""

import numpy as np
import pytest

from behavert_b200 import workloads
from behavert_b200.engine import Engine
from behavert_b200._abi import BrtError

pytestmark = pytest.mark.gpu

DT = float(np.float32(0.1))
REL = 1e-4


def _oracle():
    from oracle import oracle
    return oracle


def _targets(wl, hidden, T):
    """Final positions of a plain forward with the hidden weights."""
    with Engine(wl.params) as eng:
        eng.set_steering_weights(np.tile(np.asarray(hidden, np.float32), (len(wl.params), 1)))
        fwd = wl.meta.get("fwd_hidden", wl.fwd)
        eng.set_state(wl.pos, fwd, wl.acc)
        eng.step(DT, T)
        pos, _, _, _ = eng.get_state(features=False)
    return pos


def _min_image(d, L):
    return d - L * np.round(d / L)


def _L_per_agent(params):
    return np.concatenate([np.full(int(p.numBodies), float(p.worldSize)) for p in params])


def _counts_per_agent(params):
    return np.concatenate([np.full(int(p.numBodies), float(p.numBodies)) for p in params])


def _run(wl, target, T, k, export=True):
    eng = Engine(wl.params)
    if export:
        eng.set_option("adjoint_export", 1)
    eng.set_state(wl.pos, wl.fwd, wl.acc)
    loss = eng.adjoint_forward(target, T, k, DT)
    grads = eng.adjoint_backward()
    tape = eng.adjoint_tape(T) if export else None
    return eng, loss, grads, tape


def _reference(wl, target, tape, T):
    o = _oracle()
    lists, flags = tape
    params = wl.params
    w = np.array([[p.separationParams[0], p.alignmentParams[0], p.cohesionParams[0]] for p in params], np.float64)
    pos0, fwd0, acc0 = (a.astype(np.float64) for a in (wl.pos, wl.fwd, wl.acc))
    fin = o.frozen_forward(params, pos0, fwd0, acc0, lists, weights=w, flags=flags, dt=DT)
    L = _L_per_agent(params)[:, None]
    cnt = _counts_per_agent(params)[:, None]
    d = _min_image(fin["pos"][:, :3] - target[:, :3].astype(np.float64), L)
    gpos_T = np.zeros((len(pos0), 4))
    gpos_T[:, :3] = 2.0 * d / cnt
    rev = o.frozen_reverse(params, pos0, fwd0, acc0, lists, gpos_T, weights=w, flags=flags, dt=DT)
    f0, s0 = fwd0[:, :3], fwd0[:, 3]
    gf, gs = rev["fwd"][:, :3], rev["fwd"][:, 3]
    rev["vel"] = gs[:, None] * f0 + (gf - f0 * np.sum(f0 * gf, axis=1)[:, None]) / s0[:, None]
    loss = np.array([np.mean(np.sum(d[i:j] ** 2, axis=1)) for i, j in _ranges(params)])
    return dict(final=fin, rev=rev, loss=loss, w=w, lists=lists, flags=flags, pos0=pos0, fwd0=fwd0, acc0=acc0)


def _ranges(params):
    out, b = [], 0
    for p in params:
        out.append((b, b + int(p.numBodies)))
        b += int(p.numBodies)
    return out


def _fd_loss(wl, target, ref, *, w=None, pos=None, fwd=None):
    o = _oracle()
    fin = o.frozen_forward(wl.params, ref["pos0"] if pos is None else pos, ref["fwd0"] if fwd is None else fwd,
                           ref["acc0"], ref["lists"], weights=ref["w"] if w is None else w, flags=ref["flags"], dt=DT)
    L = _L_per_agent(wl.params)[:, None]
    d = _min_image(fin["pos"][:, :3] - target[:, :3].astype(np.float64), L)
    return sum(np.mean(np.sum(d[i:j] ** 2, axis=1)) for i, j in _ranges(wl.params))


def _check_fd(wl, target, ref, grads, n_coords, h=1e-4, seed=7, tol=REL):
    """Central differences on every weight and n_coords random state
    coordinates (positions and velocities) against the GPU gradients.
    Weights: normwise per flock; coordinates: per coordinate with an
    absolute floor of tol times the median gradient magnitude."""
    nf = len(wl.params)
    out = {"weights_fd": np.zeros((nf, 3))}
    for f in range(nf):
        for b in range(3):
            wp, wm = ref["w"].copy(), ref["w"].copy()
            wp[f, b] += h
            wm[f, b] -= h
            out["weights_fd"][f, b] = (_fd_loss(wl, target, ref, w=wp) - _fd_loss(wl, target, ref, w=wm)) / (2 * h)
        fd, g = out["weights_fd"][f], grads["weights"][f]
        assert np.linalg.norm(g - fd) <= tol * np.linalg.norm(fd), ("weights", f, g, fd)
    rng = np.random.default_rng(seed)
    n = len(ref["pos0"])
    floor = tol * np.median(np.abs(grads["pos"][:, :3]))
    worst = 0.0
    v0 = ref["fwd0"][:, :3] * ref["fwd0"][:, 3:4]
    bad = []
    for q in range(n_coords):
        i, c = int(rng.integers(n)), int(rng.integers(3))
        if q % 2 == 0:
            pp, pm = ref["pos0"].copy(), ref["pos0"].copy()
            pp[i, c] += h
            pm[i, c] -= h
            fd = (_fd_loss(wl, target, ref, pos=pp) - _fd_loss(wl, target, ref, pos=pm)) / (2 * h)
            g = grads["pos"][i, c]
        else:
            def state(e):
                v = v0[i].copy()
                v[c] += e
                f = ref["fwd0"].copy()
                s = np.linalg.norm(v)
                f[i, :3] = v / s
                f[i, 3] = s
                return f
            fd = (_fd_loss(wl, target, ref, fwd=state(h)) - _fd_loss(wl, target, ref, fwd=state(-h))) / (2 * h)
            g = grads["vel"][i, c]
        worst = max(worst, abs(g - fd) / (abs(fd) + floor))
        if not abs(g - fd) <= tol * abs(fd) + floor:
            bad.append(("pos" if q % 2 == 0 else "vel", i, c, g, fd))
    assert not bad, bad
    out["coord_worst"] = worst
    return out


def _check_reference(grads, ref, loss, tol=REL):
    """GPU gradients against the FP64 reverse: weights normwise per flock,
    position and velocity gradients normwise over all agents."""
    rev = ref["rev"]
    assert np.allclose(loss, ref["loss"], rtol=1e-5, atol=0)
    errs = {}
    gw = grads["weights"]
    for f in range(gw.shape[0]):
        e = np.linalg.norm(gw[f] - rev["weights"][f]) / np.linalg.norm(rev["weights"][f])
        errs.setdefault("weights", []).append(e)
        assert e <= tol, ("weights", f, gw[f], rev["weights"][f])
    for key in ("pos", "vel"):
        a, b = grads[key][:, :3].astype(np.float64), rev[key][:, :3]
        errs[key] = np.linalg.norm(a - b) / np.linalg.norm(b)
        assert errs[key] <= tol, (key, errs[key])
    return errs


@pytest.fixture(scope="module")
def small():
    T, k = 20, 5
    wl = workloads.adjoint(n=4096, L=40.0, steps=T)
    target = _targets(wl, wl.meta["hidden"], T)
    eng, loss, grads, tape = _run(wl, target, T, k)
    ref = _reference(wl, target, tape, T)
    yield dict(wl=wl, target=target, eng=eng, loss=loss, grads=grads, tape=tape, ref=ref, T=T, k=k)
    eng.close()


def test_taped_forward_is_the_plain_forward(small):
    wl, T = small["wl"], small["T"]
    with Engine(wl.params) as eng:
        eng.set_state(wl.pos, wl.fwd, wl.acc)
        eng.step(DT, T)
        plain = eng.get_state(features=False)
    after = small["eng"].get_state(features=False)
    for a, b in zip(plain[:3], after[:3]):
        assert np.array_equal(a, b)


def test_loss_is_fp64_mean_squared_error(small):
    wl = small["wl"]
    pos = small["eng"].get_state(features=False)[0].astype(np.float64)
    d = _min_image(pos[:, :3] - small["target"][:, :3].astype(np.float64), float(wl.params[0].worldSize))
    ref = np.mean(np.sum(d * d, axis=1))
    assert abs(small["loss"][0] - ref) <= 1e-12 * ref


def test_frozen_lists_reproduce_the_gpu_trajectory(small):
    """The exported lists and flags, replayed in FP64, follow the FP32 run."""
    wl = small["wl"]
    pos = small["eng"].get_state(features=False)[0].astype(np.float64)
    fin = small["ref"]["final"]["pos"]
    d = _min_image(fin[:, :3] - pos[:, :3], float(wl.params[0].worldSize))
    assert np.max(np.abs(d)) < 1e-3
    assert np.sqrt(np.mean(d * d)) < 1e-5


def test_gradients_match_fp64_reverse(small):
    _check_reference(small["grads"], small["ref"], small["loss"])


def test_gradients_match_central_differences(small):
    _check_fd(small["wl"], small["target"], small["ref"], small["grads"], n_coords=32)


def _same(a, b):
    a, b = np.ascontiguousarray(a), np.ascontiguousarray(b)
    return a.shape == b.shape and a.dtype == b.dtype and a.tobytes() == b.tobytes()


def test_checkpoint_interval_does_not_change_gradients(small):
    """The recomputed segments replay the forward bit for bit and the reverse
    has a fixed summation order, so the checkpoint interval changes no bit."""
    wl, target, T = small["wl"], small["target"], small["T"]
    for k in (1, 7, T):
        eng, loss, grads, _ = _run(wl, target, T, k, export=False)
        eng.close()
        assert _same(loss, small["loss"])
        for key in ("pos", "fwd", "vel", "acc", "weights"):
            assert _same(grads[key], small["grads"][key]), key


def test_backward_is_bit_reproducible(small):
    """Two engines, same state: identical loss and gradients, bit for bit
    (no float or double is accumulated with atomics)."""
    wl, target, T, k = small["wl"], small["target"], small["T"], small["k"]
    for _ in range(2):
        eng, loss, grads, _ = _run(wl, target, T, k, export=False)
        eng.close()
        assert _same(loss, small["loss"])
        for key in ("pos", "fwd", "vel", "acc", "weights"):
            assert _same(grads[key], small["grads"][key]), key


def test_repeated_backward_and_graph_reuse(small):
    wl, target, T, k = small["wl"], small["target"], small["T"], small["k"]
    eng = Engine(wl.params)
    try:
        for _ in range(2):
            eng.set_state(wl.pos, wl.fwd, wl.acc)
            loss = eng.adjoint_forward(target, T, k, DT)
            g = eng.adjoint_backward()
            assert _same(loss, small["loss"])
            assert _same(g["weights"], small["grads"]["weights"])
        g2 = eng.adjoint_backward(loss_scale=[2.0])
        assert np.allclose(g2["weights"], 2.0 * g["weights"], rtol=1e-5, atol=0)
        eng.set_option("adjoint_graphs", 0)
        eng.set_state(wl.pos, wl.fwd, wl.acc)
        loss = eng.adjoint_forward(target, T, k, DT)
        g3 = eng.adjoint_backward()
        assert _same(loss, small["loss"])
        assert _same(g3["weights"], g["weights"])
    finally:
        eng.close()


def test_extra_terminal_adjoint_matches_reference(small):
    """A terminal adjoint on the final forward and speed (no loss)."""
    o = _oracle()
    wl, target, T, k = small["wl"], small["target"], small["T"], small["k"]
    rng = np.random.default_rng(3)
    n = len(wl.pos)
    gf = np.zeros((n, 4), np.float32)
    gf[:, :4] = rng.normal(0, 1e-3, (n, 4)).astype(np.float32)
    eng = Engine(wl.params)
    try:
        eng.set_state(wl.pos, wl.fwd, wl.acc)
        eng.adjoint_forward(target, T, k, DT)
        g = eng.adjoint_backward(loss_scale=[0.0], gfwd_T=gf)
    finally:
        eng.close()
    ref = small["ref"]
    rev = o.frozen_reverse(wl.params, ref["pos0"], ref["fwd0"], ref["acc0"], ref["lists"], np.zeros((n, 4)),
                           gfwd_T=gf.astype(np.float64), weights=ref["w"], flags=ref["flags"], dt=DT)
    for key in ("pos", "fwd", "acc"):
        a, b = g[key].astype(np.float64), rev[key]
        assert np.linalg.norm(a - b) <= REL * np.linalg.norm(b), key
    assert np.all(np.abs(g["weights"] - rev["weights"]) <= REL * np.abs(rev["weights"]) + 1e-12)


def test_batched_flocks_obstacles_and_low_speed():
    """Three flocks of different sizes, sphere obstacles, speeds around the
    low-speed limit (deviation-limited steering): per-flock gradients."""
    T, k = 12, 4
    rng = np.random.default_rng(17)
    sizes = [700, 2500, 1300]
    params, pos, fwd, acc = [], [], [], []
    for f, n in enumerate(sizes):
        w = workloads.adjoint(n=n, L=32.0, steps=T, seed=30 + f)
        p = w.params[0]
        p.separationParams[0], p.alignmentParams[0], p.cohesionParams[0] = (float(x) for x in rng.uniform(0.5, 2.0, 3))
        p.numObstacles = 6
        p.obstacleAvoidanceWeight = 2.0
        for o in range(6):
            c = rng.uniform(0, 32.0, 3)
            p.obstacles[o][0], p.obstacles[o][1], p.obstacles[o][2] = (float(x) for x in c)
            p.obstacles[o][3] = float(rng.uniform(2, 5))
        wf = w.fwd.copy()
        wf[:, 3] = rng.uniform(0.05, 0.6, n).astype(np.float32)
        params.append(p)
        pos.append(w.pos)
        fwd.append(wf)
        acc.append(w.acc)
    wl = workloads.Workload("batched_adjoint", params, np.concatenate(pos), np.concatenate(fwd), np.concatenate(acc),
                            None, T, DT, {})
    target = np.concatenate(pos)[:, :3] + rng.normal(0, 1.0, (sum(sizes), 3)).astype(np.float32)
    target = np.concatenate([target, np.zeros((sum(sizes), 1), np.float32)], axis=1)
    eng, loss, grads, tape = _run(wl, target, T, k)
    eng.close()
    flags = tape[1]
    assert np.any((flags[..., 0] & 3) == 3), "deviation-limited branch not exercised"
    assert np.any(flags[..., 0] & 4), "force clip not exercised"
    ref = _reference(wl, target, tape, T)
    _check_reference(grads, ref, loss)
    # pow(speed / limit, 20) in the low-speed branch: a smaller step keeps
    # the difference quotient's truncation error below the tolerance.
    _check_fd(wl, target, ref, grads, n_coords=12, h=1e-5)


def test_unsupported_configurations_are_rejected():
    wl = workloads.adjoint(n=1024, L=32.0, steps=2)
    p = wl.params[0].copy()
    p.useKnn = 1
    with Engine([p]) as eng:
        eng.set_state(wl.pos, wl.fwd, wl.acc)
        with pytest.raises(BrtError):
            eng.adjoint_forward(wl.pos, 2, 1, DT)
    with Engine(wl.params) as eng:
        with pytest.raises(BrtError):
            eng.adjoint_backward()


def _vel_grad(rev, fwd0):
    f0, s0 = fwd0[:, :3], fwd0[:, 3]
    gf, gs = rev["fwd"][:, :3], rev["fwd"][:, 3]
    return gs[:, None] * f0 + (gf - f0 * np.sum(f0 * gf, axis=1)[:, None]) / s0[:, None]


def test_config3_full_size():
    """65,536 agents, T=50, checkpoint every 10 (config 3).

    Three gradients are compared:
      g_gpu  the CUDA adjoint: FP32 arithmetic, linearised at the FP32
             trajectory the GPU stepped through;
      g_at   the FP64 reverse linearised at that same FP32 trajectory
             (brt_adjoint_get_tape_states), seeded from the GPU's final state;
      g_64   the FP64 reverse of the FP64 frozen model (its own trajectory),
             which FP64 central differences check.
    (a) g_gpu vs g_at isolates the adjoint's own FP32 arithmetic: <= 1e-4 on
        the three weights (normwise), on the whole position and velocity
        gradients (normwise) and on 64 sampled state coordinates.
    (b) g_64 vs central differences at h = 1e-6 (h = 1e-4 carries percent-level
        truncation error at this horizon): <= 1e-4 on the weights and on the
        64 coordinates, so the FP64 model and its reverse are right.
    (c) g_at vs g_64 is the effect of the FP32 forward's rounding on the
        linearisation point, the floor of any gradient of the FP32 forward
        against the FP64 model; the GPU's distance to central differences is
        checked against it (no more than that floor plus 1e-4)."""
    o = _oracle()
    wl = workloads.adjoint()
    T, k = wl.steps, wl.meta["checkpoint_every"]
    target = _targets(wl, wl.meta["hidden"], T)
    eng = Engine(wl.params)
    try:
        eng.set_option("adjoint_export", 1)
        eng.set_state(wl.pos, wl.fwd, wl.acc)
        loss = eng.adjoint_forward(target, T, k, DT)
        grads = eng.adjoint_backward()
        lists, flags = eng.adjoint_tape(T)
        states = eng.adjoint_tape_states(T)
        final = eng.get_state(features=False)[0].astype(np.float64)
    finally:
        eng.close()
    ref = _reference(wl, target, (lists, flags), T)
    rev = ref["rev"]
    assert np.allclose(loss, ref["loss"], rtol=1e-5, atol=0)
    n = len(ref["pos0"])
    L = float(wl.params[0].worldSize)
    d32 = _min_image(final[:, :3] - target[:, :3].astype(np.float64), L)
    gT = np.zeros((n, 4))
    gT[:, :3] = 2.0 * d32 / n
    at = o.frozen_reverse_at(wl.params, states, lists, gT, weights=ref["w"], flags=flags, dt=DT)
    at["vel"] = _vel_grad(at, ref["fwd0"])

    def nrel(a, b):
        return float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b))

    report = {"weights_gpu_vs_at": nrel(grads["weights"][0], at["weights"][0]),
              "weights_at_vs_64": nrel(at["weights"][0], rev["weights"][0]),
              "weights_gpu_vs_64": nrel(grads["weights"][0], rev["weights"][0])}
    for key in ("pos", "vel"):
        report[key + "_gpu_vs_at"] = nrel(grads[key][:, :3], at[key][:, :3])
        report[key + "_at_vs_64"] = nrel(at[key][:, :3], rev[key][:, :3])
    # central differences of the FP64 model at h = 1e-6
    h = 1e-6
    fdw = np.zeros(3)
    for b in range(3):
        wp, wm = ref["w"].copy(), ref["w"].copy()
        wp[0, b] += h
        wm[0, b] -= h
        fdw[b] = (_fd_loss(wl, target, ref, w=wp) - _fd_loss(wl, target, ref, w=wm)) / (2 * h)
    report["weights_64_vs_fd"] = nrel(rev["weights"][0], fdw)
    report["weights_gpu_vs_fd"] = nrel(grads["weights"][0], fdw)
    rng = np.random.default_rng(7)
    v0 = ref["fwd0"][:, :3] * ref["fwd0"][:, 3:4]
    floor_p = 1e-4 * np.median(np.abs(at["pos"][:, :3]))
    floor_v = 1e-4 * np.median(np.abs(at["vel"][:, :3]))
    worst = {"arith": 0.0, "model": 0.0}
    for q in range(64):
        i, c = int(rng.integers(n)), int(rng.integers(3))
        if q % 2 == 0:
            pp, pm = ref["pos0"].copy(), ref["pos0"].copy()
            pp[i, c] += h
            pm[i, c] -= h
            fd = (_fd_loss(wl, target, ref, pos=pp) - _fd_loss(wl, target, ref, pos=pm)) / (2 * h)
            g, a, r, fl = grads["pos"][i, c], at["pos"][i, c], rev["pos"][i, c], floor_p
        else:
            def state(e):
                v = v0[i].copy()
                v[c] += e
                f = ref["fwd0"].copy()
                s = np.linalg.norm(v)
                f[i, :3] = v / s
                f[i, 3] = s
                return f
            fd = (_fd_loss(wl, target, ref, fwd=state(h)) - _fd_loss(wl, target, ref, fwd=state(-h))) / (2 * h)
            g, a, r, fl = grads["vel"][i, c], at["vel"][i, c], rev["vel"][i, c], floor_v
        worst["arith"] = max(worst["arith"], abs(g - a) / (abs(a) + fl))
        worst["model"] = max(worst["model"], abs(r - fd) / (abs(fd) + fl))
    report["coords_gpu_vs_at_worst"] = worst["arith"]
    report["coords_64_vs_fd_worst"] = worst["model"]
    print("config3 adjoint accuracy:", report)
    # (a) the adjoint's own arithmetic
    assert report["weights_gpu_vs_at"] <= REL
    assert report["pos_gpu_vs_at"] <= REL and report["vel_gpu_vs_at"] <= REL
    assert worst["arith"] <= REL
    # (b) the FP64 model and its reverse
    assert report["weights_64_vs_fd"] <= REL and worst["model"] <= REL
    # (c) the GPU against central differences, within the FP32-trajectory floor
    assert report["weights_gpu_vs_fd"] <= report["weights_at_vs_64"] + REL
