"""The CPU oracle against the reference's own code, compiled on the host.

oracle/build_ref.py compiles the reference's device functions of this path
with g++ from the BehaveRT sources (calcGridPos / calcGridHash,
checkForNeighbor / checkForNeighborsInCell, inBoidNeighborhood,
calcSeparation / calcAlignment / calcCohesion, adjustRawSteeringForce,
truncateLength, applySteeringForceSingle), with host stand-ins for the CUDA
keywords and textures.  This test feeds them the oracle's sorted arrays and
checks, bit for bit, on agents whose 27 cells lie inside the grid (the
reference's grid is the clamped non-periodic box; the oracle's is periodic):

  * every agent's cell hash;
  * every neighbour list: count, entries and order (the visit order and the
    maxNeighbors cap, first-M or kNN replace-farthest);
  * the flocking demo's steering force (separation, alignment, cohesion);
  * the integrated position, forward, speed and smoothed acceleration.

The reference sources are needed to build the library; without them the test
is skipped.
"""
import ctypes as C

import numpy as np
import pytest

from behavert_b200 import workloads
from oracle import build_ref, oracle


class World(C.Structure):
    _fields_ = [("gridSize", C.c_uint32), ("cellSize", C.c_float), ("maxBodiesPerCell", C.c_uint32),
                ("maxNeighbors", C.c_uint32), ("useKnn", C.c_uint32), ("searchRadius", C.c_float),
                ("maxSpeed", C.c_float), ("maxForce", C.c_float), ("mass", C.c_float),
                ("sensingMinRadius", C.c_float), ("separation", C.c_float * 3), ("alignment", C.c_float * 3),
                ("cohesion", C.c_float * 3)]


@pytest.fixture(scope="module")
def ref():
    path = build_ref.build()
    if path is None:
        pytest.skip("reference sources not available")
    L = C.CDLL(str(path))
    vp = C.c_void_p
    L.brt_ref_setup.argtypes = [C.POINTER(World), vp, vp, vp, vp]
    L.brt_ref_neighbors.argtypes = [C.c_uint32, vp, vp]
    L.brt_ref_steer.argtypes = [C.c_uint32, vp, C.c_uint32, vp]
    L.brt_ref_integrate.argtypes = [vp, C.c_float, vp, vp, vp, vp]
    L.brt_ref_adjust.argtypes = [vp, C.c_float, vp, C.c_float, vp]
    L.brt_ref_hash.argtypes = [vp]
    L.brt_ref_hash.restype = C.c_uint32
    return L


def _p(a):
    return C.c_void_p(a.ctypes.data)


def _bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def _scenario(name):
    d = oracle.params_default
    if name == "config0":
        w = workloads.plain(defaults=d)
    elif name == "dense":
        # dense Gaussian blobs: lists reach the cap of 32, so the order of the
        # 27-cell visit decides which neighbours are kept
        w = workloads.large(n=32768, defaults=d)
    elif name == "knn":
        w = workloads.plain(n=6000, L=40.0, M=6, seed=41, defaults=d)
        w.params[0].useKnn = 1
    elif name == "low_speed":
        # speeds below 0.2 * maxSpeed: adjustRawSteeringForce's deviation
        # limit, where the reference calls powf(range, 20)
        w = workloads.plain(n=4096, seed=43, defaults=d)
        rng = np.random.default_rng(43)
        w.fwd[:, 3] = rng.uniform(0.01, 0.2, n := w.num_agents).astype(np.float32)
    elif name == "minradius_cos":
        w = workloads.plain(n=4000, L=40.0, M=12, seed=42, defaults=d)
        p = w.params[0]
        p.commonSensingMinRadius = 0.5
        p.separationParams[2] = 0.2
        p.alignmentParams[1] = 3.0
        p.cohesionParams[2] = -0.5
    else:
        raise ValueError(name)
    return w


@pytest.mark.parametrize("name", ["config0", "dense", "knn", "minradius_cos", "low_speed"])
def test_oracle_matches_reference_functions(ref, name):
    w = _scenario(name)
    prm = w.params[0]
    n = w.num_agents
    G = int(round(prm.worldSize / prm.cellSize))
    M = int(prm.maxNeighbors)
    o = oracle.step(w.params, w.pos, w.fwd, w.acc, w.feat, dt=w.dt, mode=0)
    keys, ids = o["keys"], o["ids"]
    posS = np.ascontiguousarray(w.pos[ids])
    fwdS = np.ascontiguousarray(w.fwd[ids])
    occupancy = int(np.bincount(keys, minlength=G ** 3).max())
    cap = occupancy + 1
    pairs = np.full((n + cap, 2), 0xFFFFFFFF, np.uint32)  # tail: a hash no cell has
    pairs[:n, 0], pairs[:n, 1] = keys, ids
    cell_start = np.ascontiguousarray(o["cell_start"])
    world = World(G, prm.cellSize, cap, M, int(prm.useKnn), prm.commonSearchRadius, prm.commonMaxSpeed,
                  prm.commonMaxForce, prm.commonMass, prm.commonSensingMinRadius,
                  (C.c_float * 3)(*prm.separationParams), (C.c_float * 3)(*prm.alignmentParams),
                  (C.c_float * 3)(*prm.cohesionParams))
    ref.brt_ref_setup(C.byref(world), _p(cell_start), _p(pairs), _p(posS), _p(fwdS))

    # cell hash of every agent (positions lie in [0, L): the clamp never acts)
    hashes = np.array([ref.brt_ref_hash(_p(np.ascontiguousarray(w.pos[a]))) for a in range(n)], np.uint32)
    assert np.array_equal(hashes[ids], keys)

    g = np.floor(posS[:, :3] / prm.cellSize).astype(np.int64)
    interior = np.nonzero(np.all((g >= 1) & (g <= G - 2), axis=1))[0]
    assert len(interior) > n // 4
    lst = np.zeros(M, np.uint32)
    cnt = C.c_uint32()
    steer = np.zeros(3, np.float32)
    checked = full = limited = 0
    adj = np.zeros(3, np.float32)
    for i in interior:
        i = int(i)
        ref.brt_ref_neighbors(i, _p(lst), C.byref(cnt))
        k = cnt.value
        assert k == o["lists"][i, 0], (name, i)
        assert np.array_equal(lst[:k], o["lists"][i, 1:1 + k]), (name, i)
        full += int(k == M)
        ref.brt_ref_steer(i, _p(lst), k, _p(steer))
        assert np.array_equal(_bits(steer), _bits(o["steer"][i, :3])), (name, i, steer, o["steer"][i])
        a = int(ids[i])
        ref.brt_ref_adjust(_p(steer), C.c_float(float(w.fwd[a, 3])), _p(np.ascontiguousarray(w.fwd[a, :3])),
                           C.c_float(prm.commonMaxSpeed), _p(adj))
        limited += int(not np.array_equal(adj, steer))
        speed = C.c_float(float(w.fwd[a, 3]))
        fw = np.ascontiguousarray(w.fwd[a, :3])
        ps = np.ascontiguousarray(w.pos[a, :3])
        ac = np.ascontiguousarray(w.acc[a, :3])
        ref.brt_ref_integrate(_p(steer), C.c_float(w.dt), C.byref(speed), _p(fw), _p(ps), _p(ac))
        assert np.array_equal(_bits(ps), _bits(o["pos"][a, :3])), (name, a)
        assert np.array_equal(_bits(fw), _bits(o["fwd"][a, :3])), (name, a)
        assert _bits(np.float32(speed.value)) == _bits(o["fwd"][a, 3]), (name, a)
        assert np.array_equal(_bits(ac), _bits(o["acc"][a, :3])), (name, a)
        checked += 1
    print("%s: %d interior agents bit-exact, %d with a full list, %d deviation-limited" % (name, checked, full, limited))
    if name == "dense":
        assert full > 100
    if name == "low_speed":
        assert limited > 100


@pytest.mark.parametrize("name", ["plain_m15", "dense_m31"])
def test_oracle_matches_reference_kernels_for_a_whole_frame(ref, name):
    """One frame of the flocking demo through the reference's own kernels
    (genericCalcNeighgborhoodD, genericSeparationD / AlignmentD / CohesionD
    on the double-buffered force, genericApplySteeringForceD), run on the
    host agent by agent, against one oracle step.  maxNeighbors is 15 or 31:
    at those sizes the reference's list reader (uint4 words) and writer
    (stride maxNeighbors + 1) agree, so its whole chain is well defined; at
    other sizes the reader is misaligned, which the oracle does not copy."""
    d = oracle.params_default
    if name == "plain_m15":
        w = workloads.plain(M=15, seed=11, defaults=d)
    else:
        w = workloads.large(n=32768, M=31, seed=12, defaults=d)
    prm = w.params[0]
    n = w.num_agents
    G = int(round(prm.worldSize / prm.cellSize))
    M = int(prm.maxNeighbors)
    o = oracle.step(w.params, w.pos, w.fwd, w.acc, w.feat, dt=w.dt, mode=0)
    keys, ids = o["keys"], o["ids"]
    posS = np.ascontiguousarray(w.pos[ids])
    fwdS = np.ascontiguousarray(w.fwd[ids])
    accS = np.ascontiguousarray(w.acc[ids])
    cap = int(np.bincount(keys, minlength=G ** 3).max()) + 1
    pairs = np.full((n + cap, 2), 0xFFFFFFFF, np.uint32)
    pairs[:n, 0], pairs[:n, 1] = keys, ids
    cell_start = np.ascontiguousarray(o["cell_start"])
    world = World(G, prm.cellSize, cap, M, 0, prm.commonSearchRadius, prm.commonMaxSpeed, prm.commonMaxForce,
                  prm.commonMass, prm.commonSensingMinRadius, (C.c_float * 3)(*prm.separationParams),
                  (C.c_float * 3)(*prm.alignmentParams), (C.c_float * 3)(*prm.cohesionParams))
    ref.brt_ref_setup(C.byref(world), _p(cell_start), _p(pairs), _p(posS), _p(fwdS))
    lists = np.zeros((n, M + 1), np.uint32)
    pos_out = np.zeros((n, 4), np.float32)
    fwd_out = np.zeros((n, 4), np.float32)
    acc_out = np.zeros((n, 4), np.float32)
    ref.brt_ref_frame.argtypes = [C.c_uint32, C.c_float] + [C.c_void_p] * 9
    ref.brt_ref_frame(n, w.dt, _p(cell_start), _p(pairs), _p(posS), _p(fwdS), _p(accS), _p(lists), _p(pos_out),
                      _p(fwd_out), _p(acc_out))
    g = np.floor(posS[:, :3] / prm.cellSize).astype(np.int64)
    interior = np.all((g >= 1) & (g <= G - 2), axis=1)
    cnt = lists[:, 0]
    assert np.array_equal(cnt[interior], o["lists"][interior, 0])
    mask = (np.arange(M)[None, :] < cnt[:, None]) & interior[:, None]
    assert np.array_equal(np.where(mask, lists[:, 1:], 0), np.where(mask, o["lists"][:, 1:], 0))
    agents = ids[interior]
    for name_, a, b in (("pos", pos_out, o["pos"]), ("fwd", fwd_out, o["fwd"]), ("acc", acc_out, o["acc"])):
        assert np.array_equal(_bits(a[agents]), _bits(b[agents])), name_
    full = int(np.sum(cnt[interior] == M))
    print("%s: %d interior agents, lists and new state bit-exact, %d full lists" % (name, int(interior.sum()), full))
