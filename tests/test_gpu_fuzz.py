"""Randomised parity sweep: seeded random configurations, each stepped twice
on the GPU and checked against the FP32 oracle fed the same state (sorted
hashes, agent order, cell ranges, neighbour lists and the FP32 state, all
bit-exact).  The draws mix what the hand-written cases cover one at a time:
1 to 3 flocks of 1 to 3,000 agents in cubes of 3 to 11 cells a side (and
batches of 4 to 48 flocks, and flocks with their own cell sizes),
maxNeighbors from 1 to 40, kNN and first-M flocks side by side, a per-cell
cap, the 2D projection, features with and without relaxation, sphere
obstacles, a sensing minimum radius and angle cuts, dense clumps, coincident
agents and speeds down into the low-speed branch.  The same for the
Schooling law (random zones, limits, weights, speed and random deviation)
and for the crowd order run stage by stage.  Further draws run every scan
loop, and random draws of every launch option, against the default options
(bit-identical lists and state)."""
import numpy as np
import pytest

from behavert_b200.workloads import Workload, _agents, _below, _flock_params
from oracle import oracle
from tests.test_gpu_parity import _same_bits, check_step, make_engine

pytestmark = pytest.mark.gpu

DT = float(np.float32(0.1))


def _random_workload(seed: int, flocks=None, max_agents: int = 3000, cells: bool = False) -> Workload:
    """`flocks`: (low, high) bounds of the flock count, drawn uniformly;
    1 to 3 (1 twice as likely) otherwise.  `cells`: each flock draws its cell
    size (powers of two and others) and 3 to 11 cells a side; cell 4
    otherwise."""
    rng = np.random.default_rng(5000 + seed)
    nflocks = int(rng.choice([1, 1, 2, 3])) if flocks is None else int(rng.integers(flocks[0], flocks[1] + 1))
    F = int(rng.choice([0, 0, 4, 8]))
    relax = float(rng.choice([0.0, 0.05]))
    params, pos, fwd, feat = [], [], [], []
    for _ in range(nflocks):
        cell = float(rng.choice([2.0, 2.5, 3.0, 4.0, 5.0, 8.0])) if cells else 4.0
        L = cell * int(rng.integers(3, 12))
        n = int(rng.integers(1, max_agents))
        M = int(rng.choice([1, 4, 16, 32, 40]))
        p = _flock_params(n, L, M, weights=tuple(float(w) for w in rng.uniform(0.2, 2.0, 3)), F=F, relax=relax)
        p.cellSize = cell
        p.useKnn = int(rng.random() < 0.3)
        if rng.random() < 0.25:
            p.maxBodiesPerCell = int(rng.integers(1, 6))
        if rng.random() < 0.2:
            p.use2DProjection = 1
        if rng.random() < 0.3:
            p.commonSensingMinRadius = float(rng.uniform(0.0, 1.5))
            for arr in (p.separationParams, p.alignmentParams, p.cohesionParams):
                arr[1] = float(rng.uniform(1.0, 4.0))
                arr[2] = float(rng.choice([-2.0, float(rng.uniform(-1.0, 0.8))]))
        if rng.random() < 0.3:
            k = int(rng.integers(1, 8))
            p.numObstacles = k
            p.obstacleAvoidanceWeight = float(rng.uniform(0.5, 3.0))
            for o in range(k):
                c = rng.uniform(0.0, L, 3)
                p.obstacles[o][0], p.obstacles[o][1], p.obstacles[o][2] = (float(x) for x in c)
                p.obstacles[o][3] = float(rng.uniform(0.5, 4.0))
        P, W = _agents(rng, n, L)
        if n > 10 and rng.random() < 0.4:
            # a dense clump around one point, and a few agents on one spot
            m = n // 3
            P[:m, :3] = _below(rng.uniform(0, L, 3) + rng.normal(0.0, 1.5, (m, 3)), L)
            P[m:m + 3, :3] = P[0, :3]
        W[:, 3] = rng.uniform(0.05, 1.0, n).astype(np.float32)
        if p.use2DProjection:
            P[:, 1] = 0.5
        params.append(p)
        pos.append(P)
        fwd.append(W)
        if F:
            feat.append(rng.random((n, F)).astype(np.float32))
    P = np.concatenate(pos)
    W = np.concatenate(fwd)
    return Workload("fuzz", params, P, W, np.zeros_like(P), np.concatenate(feat) if F else None, 2, DT,
                    {"seed": seed})


@pytest.mark.parametrize("seed", range(80))
def test_random_configuration_two_steps(seed):
    w = _random_workload(seed)
    with make_engine(w) as eng:
        for _ in range(2):
            check_step(eng, w.params, dt=DT, fp64=False)


@pytest.mark.parametrize("seed", range(24))
def test_random_cell_sizes_two_steps(seed):
    """1 to 6 flocks, each with its own cell size: a power-of-two cell takes
    positions to cell units by its exact reciprocal, any other by the IEEE
    quotient, in one engine; a search radius of 4 may exceed the cell (both
    sides then scan the same 27 cells)."""
    w = _random_workload(900 + seed, flocks=(1, 6), max_agents=1500, cells=True)
    with make_engine(w) as eng:
        for _ in range(2):
            check_step(eng, w.params, dt=DT, fp64=False)


@pytest.mark.parametrize("seed", range(24))
def test_random_batch_of_many_flocks_two_steps(seed):
    """4 to 48 flocks of 1 to 800 agents in one engine (the batched path:
    per-flock cell bases, parameters and list modes side by side)."""
    w = _random_workload(600 + seed, flocks=(4, 48), max_agents=800)
    with make_engine(w) as eng:
        for _ in range(2):
            check_step(eng, w.params, dt=DT, fp64=False)


def _random_school(seed: int, cells: bool = False) -> Workload:
    """1 to 3 schools of one mode (an engine's flocks share the steering
    family), random zone radii, turning and blind-angle limits, weights,
    speed and random deviation; with `cells`, each school its own cell size."""
    rng = np.random.default_rng(7000 + seed)
    mode = int(rng.choice([1, 2]))
    params, pos, fwd = [], [], []
    for _ in range(int(rng.choice([1, 1, 2, 3]))):
        cell = float(rng.choice([2.0, 2.5, 3.0, 4.0, 5.0, 8.0])) if cells else 4.0
        L = cell * int(rng.integers(3, 10))
        n = int(rng.integers(2, 2500))
        p = _flock_params(n, L, int(rng.choice([4, 16, 32])))
        p.cellSize = cell
        sp = p.schooling
        sp.mode = mode
        sp.r_r = float(rng.uniform(0.3, 2.0))
        sp.r_p = float(rng.uniform(sp.r_r, 4.0))
        sp.theta = float(rng.uniform(-0.5, 0.99))
        sp.eta = float(rng.uniform(-1.0, 0.5))
        sp.w_a = float(rng.uniform(0.2, 2.0))
        sp.w_o = float(rng.uniform(1.0, 20.0))
        sp.s = float(rng.uniform(0.5, 4.0))
        sp.randomDeviationWeight = float(rng.choice([0.0, float(rng.uniform(0.0, 0.3))]))
        sp.seed = int(rng.integers(1 << 31))
        P, W = _agents(rng, n, L)
        W[:, 3] = sp.s
        if n > 10 and rng.random() < 0.4:
            m = n // 3
            P[:m, :3] = _below(rng.uniform(0, L, 3) + rng.normal(0.0, 1.0, (m, 3)), L)
        params.append(p)
        pos.append(P)
        fwd.append(W)
    P = np.concatenate(pos)
    return Workload("fuzz_school", params, P, np.concatenate(fwd), np.zeros_like(P), None, 2, DT, {"seed": seed})


@pytest.mark.parametrize("seed", range(30))
def test_random_school_two_steps(seed):
    _check_school(_random_school(seed))


@pytest.mark.parametrize("seed", range(12))
def test_random_school_cell_sizes_two_steps(seed):
    _check_school(_random_school(100 + seed, cells=True))


def _check_school(w):
    with make_engine(w) as eng:
        p, f, a = w.pos, w.fwd, w.acc
        for step in range(2):
            eng.record_lists(True)
            eng.step(DT, 1)
            lists = eng.getNeighborLists()
            pos, fwd, acc, _ = eng.get_state(features=False)
            r = oracle.step(w.params, p, f, a, dt=DT, mode=0, random_step=step + 1)
            cnt = lists[:, 0]
            assert np.array_equal(cnt, r["lists"][:, 0])
            mask = np.arange(lists.shape[1] - 1)[None, :] < cnt[:, None]
            assert np.array_equal(np.where(mask, lists[:, 1:], 0), np.where(mask, r["lists"][:, 1:], 0))
            assert _same_bits(pos, r["pos"]) and _same_bits(fwd, r["fwd"]) and _same_bits(acc, r["acc"])
            p, f, a = pos, fwd, acc


@pytest.mark.parametrize("seed", range(20))
def test_random_crowd_order_one_step(seed):
    """The crowd order, stage by stage (steerAndSlowToAvoidNeighbors, and in
    half the draws the move-away-from-base stage), on random flocks."""
    _check_crowd(_random_workload(100 + seed), seed)


@pytest.mark.parametrize("seed", range(10))
def test_random_crowd_order_cell_sizes_one_step(seed):
    _check_crowd(_random_workload(1100 + seed, cells=True), 500 + seed)


def _check_crowd(w, seed):
    for p in w.params:
        p.useKnn = 0
        p.featuresCount = 0
    w = Workload(w.name, w.params, w.pos, w.fwd, w.acc, None, 1, DT, w.meta)
    rng = np.random.default_rng(9000 + seed)
    move = None
    if rng.random() < 0.5:
        move = (tuple(float(x) for x in rng.uniform(0, 16, 3)),
                (float(rng.uniform(0.5, 3.0)), float(rng.uniform(1.0, 600.0)), float(rng.uniform(2.0, 10.0))))
    with make_engine(w) as eng:
        pos, fwd, acc, _ = eng.get_state()
        if move:
            eng.update_crowd(DT, avoid_base=move[0], avoid_base_params=move[1])
        else:
            eng.update_crowd(DT)
        lists = eng.getNeighborLists()
        gpos, gfwd, gacc, _ = eng.get_state()
    o = oracle.step(w.params, pos, fwd, acc, dt=DT, mode=0, avoid_neighbors=True, move_away=move)
    assert np.array_equal(lists[:, 0], o["lists"][:, 0])
    assert _same_bits(gpos, o["pos"]) and _same_bits(gfwd, o["fwd"]) and _same_bits(gacc, o["acc"])


def _random_adjoint(seed: int, cells: bool = False):
    """1 to 3 flocks of 200 to 3,000 agents, random weights, sometimes
    obstacles, a sensing minimum radius and angle cuts, low speeds (the
    deviation-limited branch), horizons of 4 to 12 steps with a random
    checkpoint interval, and targets near the start; with `cells`, each
    flock its own cell size."""
    rng = np.random.default_rng(11000 + seed)
    params, pos, fwd = [], [], []
    for _ in range(int(rng.choice([1, 1, 2, 3]))):
        n = int(rng.integers(200, 3000))
        cell = float(rng.choice([2.0, 2.5, 3.0, 4.0, 5.0, 8.0])) if cells else 4.0
        # the cube side of the cell-4 draws, in whole cells of the drawn
        # size, so that the density (and the conditioning of the summed
        # weight gradient) stays in the same range for every cell size
        L = cell * max(3, round(4.0 * int(rng.integers(4, 10)) / cell))
        p = _flock_params(n, L, int(rng.choice([4, 16, 32])), weights=tuple(float(w) for w in rng.uniform(0.3, 2.0, 3)))
        p.cellSize = cell
        if rng.random() < 0.3:
            p.commonSensingMinRadius = float(rng.uniform(0.0, 1.0))
            for arr in (p.separationParams, p.alignmentParams, p.cohesionParams):
                arr[1] = float(rng.uniform(2.0, 4.0))
                arr[2] = float(rng.choice([-2.0, float(rng.uniform(-0.8, 0.3))]))
        if rng.random() < 0.4:
            k = int(rng.integers(1, 6))
            p.numObstacles = k
            p.obstacleAvoidanceWeight = float(rng.uniform(0.5, 2.5))
            for o in range(k):
                c = rng.uniform(0.0, L, 3)
                p.obstacles[o][0], p.obstacles[o][1], p.obstacles[o][2] = (float(x) for x in c)
                p.obstacles[o][3] = float(rng.uniform(1.0, 4.0))
        P, W = _agents(rng, n, L)
        W[:, 3] = rng.uniform(0.05 if rng.random() < 0.5 else 0.5, 1.0, n).astype(np.float32)
        params.append(p)
        pos.append(P)
        fwd.append(W)
    P = np.concatenate(pos)
    w = Workload("fuzz_adjoint", params, P, np.concatenate(fwd), np.zeros_like(P), None, 0, DT, {})
    T = int(rng.integers(4, 13))
    k = int(rng.integers(1, T + 1))
    target = P.copy()
    target[:, :3] += rng.normal(0.0, 1.0, (len(P), 3)).astype(np.float32)
    return w, target, T, k


@pytest.mark.parametrize("seed", range(15))
def test_random_adjoint_against_fp64_reverse_at_the_gpu_trajectory(seed):
    """The GPU gradients (weights per flock, positions, velocities) against
    the FP64 frozen-neighbour reverse linearised at the GPU's own FP32
    trajectory (the adjoint's arithmetic alone), within 1e-4."""
    _check_adjoint(*_random_adjoint(seed))


@pytest.mark.parametrize("seed", range(6))
def test_random_adjoint_cell_sizes(seed):
    _check_adjoint(*_random_adjoint(100 + seed, cells=True))


def _check_adjoint(w, target, T, k):
    from tests.test_gpu_adjoint import _counts_per_agent, _L_per_agent, _min_image, _vel_grad
    with make_engine(w) as eng:
        eng.set_option("adjoint_export", 1)
        eng.set_state(w.pos, w.fwd, w.acc)
        eng.adjoint_forward(target, T, k, DT)
        g = eng.adjoint_backward()
        lists, flags = eng.adjoint_tape(T)
        states = eng.adjoint_tape_states(T)
        final = eng.get_state(features=False)[0].astype(np.float64)
    wts = np.array([[p.separationParams[0], p.alignmentParams[0], p.cohesionParams[0]] for p in w.params], np.float64)
    d = _min_image(final[:, :3] - target[:, :3].astype(np.float64), _L_per_agent(w.params)[:, None])
    gT = np.zeros((len(final), 4))
    gT[:, :3] = 2.0 * d / _counts_per_agent(w.params)[:, None]
    at = oracle.frozen_reverse_at(w.params, states, lists, gT, weights=wts, flags=flags, dt=DT)
    at["vel"] = _vel_grad(at, w.fwd.astype(np.float64))

    def nrel(a, b):
        b = np.asarray(b, np.float64)
        return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-300))

    for f in range(len(w.params)):
        assert nrel(g["weights"][f], at["weights"][f]) <= 1e-4, (f, g["weights"][f], at["weights"][f])
    assert nrel(g["pos"][:, :3], at["pos"][:, :3]) <= 1e-4
    assert nrel(g["vel"][:, :3], at["vel"][:, :3]) <= 1e-4


@pytest.mark.parametrize("seed", range(12))
def test_random_configuration_every_scan_variant(seed):
    """The random forward draws under every scan loop and list walk of the
    flock kernel: lists and state bit-identical to the default options."""
    w = _random_workload(200 + seed)

    def run(options):
        with make_engine(w) as eng:
            for k, v in options:
                eng.set_option(k, v)
            eng.record_lists(True)
            eng.step(DT, 2)
            return eng.getNeighborLists(), eng.get_state()

    ref_lists, ref = run([])
    for scan, walk in ((0, 0), (0, 1), (1, 0), (2, 1), (3, 0), (4, 0), (4, 2), (5, 0), (6, 2), (7, 2)):
        lists, out = run([("scan_variant", scan), ("phase2_variant", walk)])
        assert np.array_equal(lists[:, 0], ref_lists[:, 0]), (scan, walk)
        mask = np.arange(lists.shape[1] - 1)[None, :] < lists[:, :1]
        assert np.array_equal(np.where(mask, lists[:, 1:], 0), np.where(mask, ref_lists[:, 1:], 0)), (scan, walk)
        for a, b in zip(ref, out):
            if a is not None:
                assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), (scan, walk)


@pytest.mark.parametrize("seed", range(64))
def test_random_configuration_random_options(seed):
    """Random forward draws under a random draw of every launch option the
    autotuner and the user can set (block size, sort digit width, scan loop,
    list walk, register budget, incremental re-sort, forced two-pass kernel):
    lists and state after three steps bit-identical to the default options.
    Odd draws hold 4 to 48 flocks."""
    w = _random_workload(400 + seed, **({"flocks": (4, 48), "max_agents": 800} if seed % 2 else {}))
    rng = np.random.default_rng(12000 + seed)
    options = [
        ("block_size", int(rng.choice([32, 64, 96, 128, 160, 192, 256]))),
        ("sort_digit_bits", int(rng.integers(4, 10))),
        ("scan_variant", int(rng.integers(0, 8))),
        ("phase2_variant", int(rng.integers(0, 3))),
        ("registers", int(rng.choice([40, 48, 64, 128]))),
        ("incremental_sort", int(rng.integers(0, 2))),
        ("two_pass", int(rng.random() < 0.25)),
    ]

    def run(opts):
        with make_engine(w) as eng:
            for k, v in opts:
                eng.set_option(k, v)
            eng.record_lists(True)
            eng.step(DT, 3)
            return eng.getNeighborLists(), eng.get_state()

    ref_lists, ref = run([])
    lists, out = run(options)
    assert np.array_equal(lists[:, 0], ref_lists[:, 0]), options
    mask = np.arange(lists.shape[1] - 1)[None, :] < lists[:, :1]
    assert np.array_equal(np.where(mask, lists[:, 1:], 0), np.where(mask, ref_lists[:, 1:], 0)), options
    for a, b in zip(ref, out):
        if a is not None:
            assert _same_bits(a, b), options
