"""GPU parity tests: the CUDA path (through the C-ABI) against the CPU oracle.

Integer outputs (sorted hashes, agent order, cell ranges, neighbour lists) must
be bit-exact.  The FP32 state must be bit-identical to the FP32 oracle (same
operation order, IEEE division and square root, no contraction, and the
low-speed branch's power evaluated by the same double-precision sequence on
both sides).  Against the FP64 oracle, fed the same FP32 state, each agent's
per-step relative error must stay within the benchmark target's 1e-5 for at
least 99% of the agents (the rest are ill-conditioned in FP32 itself; the
maximum per agent and the normwise error are reported).

Horizons: config 0 is compared at every one of its 200 steps and over the
whole 200-step trajectory; config 1 at full size (1,048,576 agents) at each of
its first 10 steps (the incremental re-sort from step 2 on) and at the end of
its 100-step horizon; configs 2 and 4 at full size (10.9 M and 2.7 M agents)
at their first two steps.
"""
import numpy as np
import pytest

from behavert_b200 import Engine, workloads
from oracle import oracle

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-5       # per-step state vs FP64 oracle, per agent (relative)
MAX_FRAC_OVER = 1e-2  # fraction of agents allowed above TOL_FP64 on their own (99% within)


def _rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    scale = max(np.abs(b).max(), 1e-30)
    with np.errstate(invalid="ignore"):  # states holding inf report NaN here
        return float(np.abs(a - b).max() / scale)


def _vel(fwd):
    return fwd[:, :3].astype(np.float64) * fwd[:, 3:4].astype(np.float64)


def check_step(eng: Engine, params, dt=0.1, stats=None, full=True, fp64=True):
    """Run one fused GPU step from the engine's current state and compare it
    with the oracle fed the same state.  Returns the error summary."""
    pos, fwd, acc, feat = eng.get_state()
    if stats is None and any(p.clusteringForceParams[0] or p.alignmentClusteringForceParams[0] for p in params):
        stats = eng.get_similarity_stats()
    eng.record_lists(True)
    eng.step(dt, 1)
    keys, ids = eng.getHash()
    cs, ce = eng.getCellRanges()
    lists = eng.getNeighborLists()
    gpos, gfwd, gacc, gfeat = eng.get_state()
    o = oracle.step(params, pos, fwd, acc, feat, stats, dt=dt, mode=0)
    assert np.array_equal(keys, o["keys"]), "sorted hashes differ"
    assert np.array_equal(ids, o["ids"]), "sorted agent order differs"
    assert np.array_equal(cs, o["cell_start"]) and np.array_equal(ce, o["cell_end"]), "cell ranges differ"
    cnt = lists[:, 0]
    assert np.array_equal(cnt, o["lists"][:, 0]), "neighbour counts differ"
    M = lists.shape[1] - 1
    mask = np.arange(M)[None, :] < cnt[:, None]
    assert np.array_equal(np.where(mask, lists[:, 1:], 0), np.where(mask, o["lists"][:, 1:], 0)), "neighbour lists differ"
    err = {"pos32": _rel(gpos, o["pos"]), "vel32": _rel(_vel(gfwd), _vel(o["fwd"])), "acc32": _rel(gacc, o["acc"])}
    for name, g, r in (("pos", gpos, o["pos"]), ("fwd", gfwd, o["fwd"]), ("acc", gacc, o["acc"]),
                       ("feat", gfeat, o["feat"])):
        if g is not None:
            assert _same_bits(g, r), "FP32 %s differs from the FP32 oracle: %s" % (name, err)
    if fp64:
        o64 = oracle.step(params, pos.astype(np.float64), fwd.astype(np.float64), acc.astype(np.float64),
                          None if feat is None else feat.astype(np.float64),
                          None if stats is None else stats.astype(np.float64), dt=dt, mode=1, want_intermediates=False)
        # positions: max error relative to the world scale; velocity and
        # features: each agent's own relative error within 1e-5 for at least
        # 99% of the agents.  The FP32 step is bit-identical to the FP32
        # oracle; the agents beyond 1e-5 are ill-conditioned in FP32 itself
        # (normalize of a steering sum that nearly cancels, whose direction
        # FP32 and FP64 then take differently).  In a small flock one such
        # agent carries the normwise error of the whole state (config 0:
        # up to 4.5e-4 at its worst step, from one agent of 4,096), so the
        # normwise error and the maximum per agent are reported, not gated.
        err["pos64"] = _pos_rel(gpos, o64["pos"], params)
        err.update(_fp64_errors("vel", _vel(gfwd), _vel(o64["fwd"])))
        assert err["pos64"] <= TOL_FP64, err
        assert err["vel_over"] <= MAX_FRAC_OVER, err
        if gfeat is not None:
            err.update(_fp64_errors("feat", gfeat, o64["feat"]))
            assert err["feat_over"] <= MAX_FRAC_OVER, err
    return err


def _pos_rel(g, r, params):
    """Largest position difference, taken through the periodic wrap of each
    flock's cube, relative to the largest coordinate."""
    L = np.concatenate([np.full(int(p.numBodies), float(p.worldSize)) for p in params])[:, None]
    d = np.asarray(g, np.float64)[:, :3] - np.asarray(r, np.float64)[:, :3]
    d -= L * np.round(d / L)
    return float(np.abs(d).max() / max(np.abs(np.asarray(r, np.float64)[:, :3]).max(), 1e-30))


def _same_bits(a, b):
    """Every value bit-identical, and NaN where the other side has NaN.  The
    payload of a NaN an operation generates (0/0 of coincident agents) is left
    to the implementation by IEEE 754: the GPU gives 0x7fffffff and x86
    0xffc00000, so NaN payloads are not compared."""
    a = np.ascontiguousarray(a, np.float32)
    b = np.ascontiguousarray(b, np.float32)
    if a.shape != b.shape:
        return False
    na, nb = np.isnan(a), np.isnan(b)
    return np.array_equal(na, nb) and np.array_equal(a.view(np.uint32)[~na], b.view(np.uint32)[~nb])


def _fp64_errors(name, g, r):
    g = np.asarray(g, np.float64)
    r = np.asarray(r, np.float64)
    per = np.linalg.norm(g - r, axis=1) / np.maximum(np.linalg.norm(r, axis=1), 1e-30)
    return {name + "_l2": float(np.linalg.norm(g - r) / max(np.linalg.norm(r), 1e-30)),
            name + "_p9999": float(np.percentile(per, 99.99)), name + "_max": float(per.max()),
            name + "_over": float(np.mean(per > TOL_FP64))}


def make_engine(w):
    eng = Engine(w.params)
    eng.set_state(w.pos, w.fwd, w.acc, w.feat)
    return eng


def test_plain_config0_every_step_of_the_horizon():
    """Config 0's 200 steps, each checked against the oracle fed the GPU's
    state: lists bit-exact, FP32 state bit-identical, FP64 within 1e-5."""
    w = workloads.plain()
    worst = {}
    with make_engine(w) as eng:
        for _ in range(w.steps):
            err = check_step(eng, w.params)
            for k, v in err.items():
                worst[k] = max(worst.get(k, 0.0), v)
    print("config 0, 200 steps, worst per-step errors:", worst)


def test_plain_config0_trajectory_full_horizon():
    """The 200-step trajectory as one CUDA graph (the production path, no
    lists written) against 200 oracle steps from the same seeded state: the
    FP32 states are bit-identical at the end of the horizon."""
    w = workloads.plain()
    with make_engine(w) as eng:
        eng.step(w.dt, w.steps)
        gpos, gfwd, gacc, _ = eng.get_state()
    pos, fwd, acc = w.pos, w.fwd, w.acc
    for _ in range(w.steps):
        o = oracle.step(w.params, pos, fwd, acc, dt=w.dt, want_intermediates=False)
        pos, fwd, acc = o["pos"], o["fwd"], o["acc"]
    assert _same_bits(gpos, pos) and _same_bits(gfwd, fwd) and _same_bits(gacc, acc)


def test_large_scaled_with_features():
    w = workloads.large(n=65536)
    with make_engine(w) as eng:
        for _ in range(3):
            err = check_step(eng, w.params)
    print(err)


def test_large_full_size_first_ten_steps():
    """Config 1 at full size, steps 1-10 each against the oracle.  Step 1 takes
    the full radix sort (the state was just set); steps 2-10 take the
    incremental re-sort, so that path is pinned at 1,048,576 agents."""
    w = workloads.large()
    worst = {}
    with make_engine(w) as eng:
        for _ in range(10):
            err = check_step(eng, w.params)
            for k, v in err.items():
                worst[k] = max(worst.get(k, 0.0), v)
    print("config 1 full size, steps 1-10, worst per-step errors:", worst)


def test_large_full_size_horizon_endpoint():
    """Config 1's 100-step horizon as one CUDA graph (production path) against
    100 oracle steps from the seeded state: bit-identical FP32 state, features
    included, at the end of the horizon."""
    w = workloads.large()
    with make_engine(w) as eng:
        eng.step(w.dt, w.steps)
        g = eng.get_state()
    pos, fwd, acc, feat = w.pos, w.fwd, w.acc, w.feat
    for _ in range(w.steps):
        o = oracle.step(w.params, pos, fwd, acc, feat, dt=w.dt, want_intermediates=False)
        pos, fwd, acc, feat = o["pos"], o["fwd"], o["acc"], o["feat"]
    for name, x, y in zip(("pos", "fwd", "acc", "feat"), g, (pos, fwd, acc, feat)):
        assert _same_bits(x, y), name


def test_stagewise_equals_fused():
    w = workloads.large(n=20000)
    with make_engine(w) as a, make_engine(w) as b:
        a.record_lists(True)
        a.step(0.1, 1)
        b.update_stagewise(0.1)
        assert np.array_equal(a.getNeighborLists()[:, 0], b.getNeighborLists()[:, 0])
        sa, sb = a.get_state(), b.get_state()
        for x, y in zip(sa, sb):
            assert np.array_equal(x, y)


def test_crowd_order_steer_and_slow_to_avoid_neighbors():
    """steerAndSlowToAvoidNeighbors in the crowd sample's order, stage by
    stage through the C-ABI, against the oracle: lists bit-exact, the state
    within the FP32 / FP64 tolerances (a flipped speed branch would move an
    agent's speed by 2-10%)."""
    w = workloads.plain(n=4096, L=40.0, M=32, seed=5, steps=1)
    with make_engine(w) as eng:
        pos, fwd, acc, _ = eng.get_state()
        eng.update_crowd(w.dt)
        lists = eng.getNeighborLists()
        gpos, gfwd, gacc, _ = eng.get_state()
    o = oracle.step(w.params, pos, fwd, acc, dt=w.dt, mode=0, avoid_neighbors=True)
    cnt = lists[:, 0]
    assert np.array_equal(cnt, o["lists"][:, 0])
    assert (cnt > 18).sum() > 100 and (cnt <= 16).sum() > 100
    mask = np.arange(lists.shape[1] - 1)[None, :] < cnt[:, None]
    assert np.array_equal(np.where(mask, lists[:, 1:], 0), np.where(mask, o["lists"][:, 1:], 0))
    assert _same_bits(gpos, o["pos"]) and _same_bits(gfwd, o["fwd"]) and _same_bits(gacc, o["acc"])
    plain = oracle.step(w.params, pos, fwd, acc, dt=w.dt, mode=0)
    assert _rel(_vel(gfwd), _vel(plain["fwd"])) > 1e-4
    o64 = oracle.step(w.params, *(x.astype(np.float64) for x in (pos, fwd, acc)), dt=w.dt, mode=1,
                      want_intermediates=False, avoid_neighbors=True)
    assert _pos_rel(gpos, o64["pos"], w.params) <= TOL_FP64
    e = _fp64_errors("vel", _vel(gfwd), _vel(o64["fwd"]))
    assert e["vel_over"] <= MAX_FRAC_OVER, e


def test_crowd_order_full_size_one_step():
    """The crowd order, stage by stage, on 1,048,576 agents (the size the
    benchmark measures): lists and FP32 state bit-exact."""
    w = workloads.plain(n=1 << 20, L=256.0, M=32, seed=5, steps=1)
    with make_engine(w) as eng:
        pos, fwd, acc, _ = eng.get_state()
        eng.update_crowd(w.dt)
        lists = eng.getNeighborLists()
        gpos, gfwd, gacc, _ = eng.get_state()
    o = oracle.step(w.params, pos, fwd, acc, dt=w.dt, mode=0, avoid_neighbors=True)
    cnt = lists[:, 0]
    assert np.array_equal(cnt, o["lists"][:, 0])
    mask = np.arange(lists.shape[1] - 1)[None, :] < cnt[:, None]
    assert np.array_equal(np.where(mask, lists[:, 1:], 0), np.where(mask, o["lists"][:, 1:], 0))
    assert _same_bits(gpos, o["pos"]) and _same_bits(gfwd, o["fwd"]) and _same_bits(gacc, o["acc"])


def test_crowd_order_with_move_away_from_base():
    """The crowd order with steerForMoveAwayBaseTarget after cohesion, stage
    by stage through the C-ABI, against the oracle."""
    w = workloads.plain(n=4096, L=40.0, M=32, seed=6, steps=1)
    base, prm = (20.0, 15.0, 25.0), (2.0, 500.0, 8.0)
    with make_engine(w) as eng:
        pos, fwd, acc, _ = eng.get_state()
        eng.update_crowd(w.dt, avoid_base=base, avoid_base_params=prm)
        lists = eng.getNeighborLists()
        gpos, gfwd, gacc, _ = eng.get_state()
    o = oracle.step(w.params, pos, fwd, acc, dt=w.dt, mode=0, avoid_neighbors=True, move_away=(base, prm))
    assert np.array_equal(lists[:, 0], o["lists"][:, 0])
    assert _same_bits(gpos, o["pos"]) and _same_bits(gfwd, o["fwd"]) and _same_bits(gacc, o["acc"])
    without = oracle.step(w.params, pos, fwd, acc, dt=w.dt, mode=0, avoid_neighbors=True)
    assert _rel(_vel(gfwd), _vel(without["fwd"])) > 1e-4
    o64 = oracle.step(w.params, *(x.astype(np.float64) for x in (pos, fwd, acc)), dt=w.dt, mode=1,
                      want_intermediates=False, avoid_neighbors=True, move_away=(base, prm))
    assert _pos_rel(gpos, o64["pos"], w.params) <= TOL_FP64
    e = _fp64_errors("vel", _vel(gfwd), _vel(o64["fwd"]))
    assert e["vel_over"] <= MAX_FRAC_OVER, e


def test_single_pass_equals_two_pass():
    """The single-pass fused kernel and the list-first kernel agree bit for bit."""
    w = workloads.large(n=40000)
    with make_engine(w) as a, make_engine(w) as b:
        b.set_option("two_pass", 1)
        for eng in (a, b):
            eng.record_lists(True)
            eng.step(0.1, 3)
        assert np.array_equal(a.getNeighborLists(), b.getNeighborLists())
        for x, y in zip(a.get_state(), b.get_state()):
            assert np.array_equal(x, y)


@pytest.mark.parametrize("bits", [5, 7, 9])
def test_sort_digit_width_option(bits):
    w = workloads.large(n=30000)
    with make_engine(w) as a, make_engine(w) as b:
        b.set_option("sort_digit_bits", bits)
        a.step(0.1, 2)
        b.step(0.1, 2)
        for x, y in zip(a.get_state(), b.get_state()):
            assert np.array_equal(x, y)
        assert np.array_equal(a.getHash()[1], b.getHash()[1])


def test_graph_equals_single_steps():
    w = workloads.plain(n=8192, L=80.0)
    with make_engine(w) as a, make_engine(w) as b:
        a.step(0.1, 12)
        for _ in range(12):
            b.step(0.1, 1)
        for x, y in zip(a.get_state(), b.get_state()):
            if x is not None:
                assert np.array_equal(x, y)
        # replaying the cached graph continues from the current state
        a.step(0.1, 12)
        for _ in range(12):
            b.step(0.1, 1)
        for x, y in zip(a.get_state(), b.get_state()):
            if x is not None:
                assert np.array_equal(x, y)


def test_batched_small():
    w = workloads.batched(num_flocks=24, lo=50, hi=3000, seed=7)
    with make_engine(w) as eng:
        for _ in range(2):
            check_step(eng, w.params)


def test_batched_full_size_first_two_steps():
    """Config 2 at full size (1,024 flocks, 10.9 M agents): step 1 (full radix
    sort on the (flock, cell) key) and step 2 (incremental re-sort), lists,
    order and FP32 state bit-exact against the oracle, and within the FP64
    tolerances."""
    w = workloads.batched()
    with make_engine(w) as eng:
        for _ in range(2):
            check_step(eng, w.params)


def test_fitting_full_size_first_two_steps():
    """Config 4 at full size (256 flocks, 2.7 M agents, 32 sphere obstacles
    each): two steps against the FP32 and FP64 oracle."""
    w = workloads.fitting()
    with make_engine(w) as eng:
        for _ in range(2):
            check_step(eng, w.params)


def test_clustering_steering_and_stats():
    w = workloads.plain(n=3000, L=40.0, M=12, seed=31)
    p = w.params[0]
    p.featuresCount = 5
    p.clusteringForceParams[0] = 0.7
    p.alignmentClusteringForceParams[0] = 0.4
    p.featureRelaxRate = 0.05
    rng = np.random.default_rng(31)
    w.feat = rng.random((3000, 5)).astype(np.float32)
    stats = np.tile(np.array([0.3, 0.5, 0.7, 0.0], np.float32), (3000, 1))
    with make_engine(w) as eng:
        eng.set_similarity_stats(stats)
        for _ in range(2):
            check_step(eng, w.params)


def test_obstacles():
    w = workloads.fitting(num_flocks=3, lo=400, hi=2500, seed=8, obstacles=10)
    with make_engine(w) as eng:
        check_step(eng, w.params)


@pytest.mark.parametrize("M", [16, 40])
def test_knn_and_first_m_flocks_in_one_engine(M):
    """kNN replacement is per flock: an engine holding a useKnn flock and a
    first-M flock gives each its own lists (M <= 32: the cooperative kNN scan
    of the single-pass kernel; M > 32: the two-pass kernel), bit-exact."""
    a = workloads.plain(n=3000, L=28.0, M=M, seed=51)
    b = workloads.plain(n=2500, L=28.0, M=M, seed=52)
    a.params[0].useKnn = 1
    w = workloads.Workload("mixed", a.params + b.params, np.concatenate([a.pos, b.pos]),
                           np.concatenate([a.fwd, b.fwd]), np.concatenate([a.acc, b.acc]), None, 2, a.dt, {})
    with make_engine(w) as eng:
        for _ in range(2):
            check_step(eng, w.params)


@pytest.mark.parametrize("block", [64, 256])
def test_knn_dense_blobs_with_features(block):
    """The cooperative kNN scan where lists fill and most accepted candidates
    replace an entry (Gaussian blobs at config 1's density, 8 relaxed
    features), three steps, bit-exact lists and state."""
    w = workloads.large(n=1 << 16, steps=3)
    w.params[0].useKnn = 1
    with make_engine(w) as eng:
        eng.set_option("block_size", block)
        for _ in range(3):
            check_step(eng, w.params)


def test_knn_full_size_first_two_steps():
    """Config 1 at full size with kNN lists (the nearest 32 kept; the
    cooperative kNN scan): two steps against the FP32 and FP64 oracle."""
    w = workloads.large()
    w.params[0].useKnn = 1
    with make_engine(w) as eng:
        for _ in range(2):
            check_step(eng, w.params)


@pytest.mark.parametrize("variant", ["knn", "maxbodies", "2d", "minradius_cos"])
def test_variants(variant):
    w = workloads.plain(n=4000, L=40.0, M=6, seed=41)
    p = w.params[0]
    if variant == "knn":
        p.useKnn = 1
    elif variant == "maxbodies":
        p.maxBodiesPerCell = 2
    elif variant == "2d":
        p.use2DProjection = 1
    elif variant == "minradius_cos":
        p.commonSensingMinRadius = 0.5
        p.separationParams[2] = 0.2
        p.alignmentParams[1] = 3.0
        p.cohesionParams[2] = -0.5
    with make_engine(w) as eng:
        check_step(eng, w.params, fp64=variant != "2d")


def test_edge_cases_dense_boundary_frozen():
    n = 300
    w = workloads.plain(n=n, L=16.0, M=40, seed=3)
    rng = np.random.default_rng(3)
    # everyone in one corner cell wrapping around the boundary, some exactly on faces
    w.pos[:, :3] = (rng.random((n, 3)) * 1.5).astype(np.float32)
    w.pos[:50, 0] = 0.0
    w.pos[50:60, :3] = np.nextafter(np.float32(16.0), np.float32(0))
    w.fwd[:5, 3] = -1.0  # frozen agents (speed < 0)
    with make_engine(w) as eng:
        check_step(eng, w.params, fp64=False)


@pytest.mark.parametrize("cell,G", [(2.0, 8), (8.0, 4), (3.0, 5), (2.5, 6)])
def test_cell_sizes(cell, G):
    """Cell sizes other than 4: a power-of-two cell takes its position to
    cell units by the exact reciprocal, any other by the IEEE quotient; both
    hash, list and step as the oracle's division does."""
    w = workloads.plain(n=1500, L=cell * G, M=16, seed=9)
    p = w.params[0]
    p.cellSize = cell
    p.commonSearchRadius = min(4.0, cell)
    w.pos[:20, 0] = np.float32(cell) * np.arange(20, dtype=np.float32) % np.float32(cell * G)  # on cell faces
    with make_engine(w) as eng:
        for _ in range(2):
            check_step(eng, w.params, fp64=False)


def _non_finite_workload(seed):
    """Positions a neighbour-cell cull must not trust: NaN agents (every axis,
    and one axis only) hashed into cell 0 beside finite agents there, infinite
    coordinates, agents outside the world clamped into edge cells (some past
    the int range of the cell conversion).  A NaN candidate passes the radius
    test (!(NaN > r)) of every agent that reads its cell; a NaN agent accepts
    every candidate it reads."""
    n = 600
    w = workloads.plain(n=n, L=16.0, M=40, seed=seed)
    rng = np.random.default_rng(seed)
    w.pos[:40, :3] = (rng.random((40, 3)) * 3.0).astype(np.float32)
    w.pos[40:43, :3] = np.nan
    w.pos[43, 0] = np.nan
    w.pos[44, 1] = np.inf
    w.pos[45, 2] = -np.inf
    w.pos[46, 0] = -3.0
    w.pos[47, 0] = 21.0
    w.pos[48, 1] = 17.5
    w.pos[49, 2] = 1e30   # past the int range: the device conversion saturates (last cell)
    w.pos[50, 0] = -1e30
    return w


@pytest.mark.parametrize("scan,walk", [(0, 0), (1, 0), (2, 1), (3, 0), (4, 0), (5, 2), (6, 2), (7, 2)])
def test_non_finite_and_outside_positions_every_scan(scan, walk):
    """Every scan loop against the oracle on such a state, two steps (the
    NaN spreads to the neighbours in the first)."""
    w = _non_finite_workload(7)
    with make_engine(w) as eng:
        eng.set_option("scan_variant", scan)
        eng.set_option("phase2_variant", walk)
        for _ in range(2):
            check_step(eng, w.params, fp64=False)


@pytest.mark.parametrize("M", [16, 40])
def test_non_finite_and_outside_positions_knn(M):
    """kNN lists on the same state: the cooperative kNN scan (maxNeighbors up
    to a warp) and the two-pass kernel above it.  A NaN distance fills a free
    list entry but never displaces a kept one (dist < maxDistValue fails)."""
    w = _non_finite_workload(7)
    w.params[0].useKnn = 1
    w.params[0].maxNeighbors = M
    with make_engine(w) as eng:
        for _ in range(2):
            check_step(eng, w.params, fp64=False)


def test_non_finite_and_outside_positions_crowd_order():
    """The stage-wise crowd order on the same state."""
    w = _non_finite_workload(7)
    with make_engine(w) as eng:
        pos, fwd, acc, _ = eng.get_state()
        eng.update_crowd(w.dt)
        lists = eng.getNeighborLists()
        gpos, gfwd, gacc, _ = eng.get_state()
    o = oracle.step(w.params, pos, fwd, acc, dt=w.dt, mode=0, avoid_neighbors=True)
    cnt = lists[:, 0]
    assert np.array_equal(cnt, o["lists"][:, 0])
    mask = np.arange(lists.shape[1] - 1)[None, :] < cnt[:, None]
    assert np.array_equal(np.where(mask, lists[:, 1:], 0), np.where(mask, o["lists"][:, 1:], 0))
    assert _same_bits(gpos, o["pos"]) and _same_bits(gfwd, o["fwd"]) and _same_bits(gacc, o["acc"])


def test_single_agent_and_tiny_flock():
    w = workloads.plain(n=1, L=12.0, M=4, seed=2)
    with make_engine(w) as eng:
        check_step(eng, w.params)
        assert eng.getNeighborLists()[0, 0] == 0
