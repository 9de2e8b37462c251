"""CPU tests of the oracle: independent numpy restatement, known-answer cases,
sort/cell-range invariants, FP32-vs-FP64 error and the committed golden
fixtures (regression pins of the oracle's own outputs)."""
from pathlib import Path

import numpy as np
import pytest

from behavert_b200 import workloads
from oracle import oracle
from tests.brute import grid_coord, lists_bruteforce

GOLDEN = Path(__file__).resolve().parent / "golden"


def _small(n=600, L=32.0, M=8, seed=11):
    w = workloads.plain(n=n, L=L, M=M, seed=seed)
    return w


def _sorted_state(o, w):
    return w.pos[o["ids"]]


def test_hash_sort_and_cell_ranges():
    w = _small()
    o = oracle.step(w.params, w.pos, w.fwd, w.acc, dt=0.1)
    G = int(w.params[0].worldSize / w.params[0].cellSize)
    g = grid_coord(w.pos[:, :3], 4.0, G)
    keys = (g[:, 2] * G + g[:, 1]) * G + g[:, 0]
    order = np.lexsort((np.arange(len(keys)), keys))  # stable: key, then id
    assert np.array_equal(o["ids"], order)
    assert np.array_equal(o["keys"], keys[order])
    cs, ce = o["cell_start"], o["cell_end"]
    for c in range(G ** 3):
        idx = np.nonzero(o["keys"] == c)[0]
        if len(idx) == 0:
            assert cs[c] == 0xFFFFFFFF and ce[c] == 0xFFFFFFFF
        else:
            assert cs[c] == idx[0] and ce[c] == idx[-1] + 1


@pytest.mark.parametrize("M", [3, 8, 40])
def test_lists_match_bruteforce(M):
    w = _small(n=400, L=24.0, M=M, seed=5)
    o = oracle.step(w.params, w.pos, w.fwd, w.acc, dt=0.1)
    ref = lists_bruteforce(_sorted_state(o, w), 24.0, 4.0, 4.0, M)
    lists = o["lists"]
    for i, r in enumerate(ref):
        n = lists[i, 0]
        assert n == len(r), i
        assert list(lists[i, 1:1 + n]) == r, i


def test_lists_bruteforce_grid3_wrap():
    # G = 3: every cell is adjacent to every other through a wrap.
    w = _small(n=120, L=12.0, M=10, seed=9)
    o = oracle.step(w.params, w.pos, w.fwd, w.acc, dt=0.1)
    ref = lists_bruteforce(_sorted_state(o, w), 12.0, 4.0, 4.0, 10)
    for i, r in enumerate(ref):
        assert list(o["lists"][i, 1:1 + o["lists"][i, 0]]) == r


def _kat(positions, L=16.0, M=4, radius=4.0):
    n = len(positions)
    w = workloads.plain(n=n, L=L, M=M, seed=0)
    p = w.params[0]
    p.commonSearchRadius = radius
    pos = np.zeros((n, 4), np.float32)
    pos[:, :3] = np.asarray(positions, np.float32)
    pos[:, 3] = 1
    fwd = np.zeros((n, 4), np.float32)
    fwd[:, 0] = 1
    fwd[:, 3] = 0.75
    acc = np.zeros((n, 4), np.float32)
    return oracle.step([p], pos, fwd, acc, dt=0.1), w


def _list_of_agent(o, agent):
    slot = int(np.nonzero(o["ids"] == agent)[0][0])
    n = o["lists"][slot, 0]
    return sorted(int(o["ids"][s]) for s in o["lists"][slot, 1:1 + n])


def test_kat_radius_boundary_inclusive():
    # exactly 4.0 apart: sqrtf(16) == 4 is not > 4 -> neighbours
    o, _ = _kat([[5.0, 5.0, 5.0], [9.0, 5.0, 5.0]])
    assert _list_of_agent(o, 0) == [1]
    assert _list_of_agent(o, 1) == [0]
    # one ulp beyond
    far = np.nextafter(np.float32(9.0), np.float32(10.0))
    o, _ = _kat([[5.0, 5.0, 5.0], [far, 5.0, 5.0]])
    assert _list_of_agent(o, 0) == []


def test_kat_periodic_wrap():
    # across the x boundary of a 16-cube: 0.5 and 15.5 are 1.0 apart
    o, _ = _kat([[0.5, 8.0, 8.0], [15.5, 8.0, 8.0], [8.0, 8.0, 8.0]])
    assert _list_of_agent(o, 0) == [1]
    assert _list_of_agent(o, 1) == [0]
    assert _list_of_agent(o, 2) == []
    # corner wrap in all three axes
    o, _ = _kat([[0.2, 0.2, 0.2], [15.9, 15.9, 15.9]])
    assert _list_of_agent(o, 0) == [1]


def test_kat_cap_keeps_visit_order():
    # home agent at the centre of a cell, neighbours in cells with offsets
    # x=-1 (visited first), x=0 and x=+1; M=2 keeps the first two in visit order
    centre = [6.0, 6.0, 6.0]
    pts = [centre, [8.5, 6.0, 6.0], [3.5, 6.0, 6.0], [6.5, 6.0, 6.0], [2.5, 6.0, 6.2]]
    o, _ = _kat(pts, M=2)
    # visit order: x-1 cell holds agents 2 (x=3.5) and 4 (x=4.5) -> both, by slot
    assert _list_of_agent(o, 0) == [2, 4]


def test_kat_duplicate_positions():
    o, _ = _kat([[6.0, 6.0, 6.0], [6.0, 6.0, 6.0]])
    assert _list_of_agent(o, 0) == [1]
    # inBoidNeighborhood rejects a zero offset (normalize(0) is NaN), so no
    # steering term and no NaN in the new state
    assert np.all(np.isfinite(o["pos"])) and np.all(np.isfinite(o["fwd"]))


def test_fp32_vs_fp64_per_step():
    w = workloads.plain()
    o32 = oracle.step(w.params, w.pos, w.fwd, w.acc, dt=0.1, mode=0, want_intermediates=False)
    o64 = oracle.step(w.params, w.pos.astype(np.float64), w.fwd.astype(np.float64), w.acc.astype(np.float64),
                      dt=0.1, mode=1, want_intermediates=False)
    rel_pos = np.abs(o32["pos"] - o64["pos"]).max() / np.abs(o64["pos"]).max()
    vel32 = o32["fwd"][:, :3].astype(np.float64) * o32["fwd"][:, 3:4]
    vel64 = o64["fwd"][:, :3] * o64["fwd"][:, 3:4]
    rel_vel = np.abs(vel32 - vel64).max() / np.abs(vel64).max()
    assert rel_pos < 1e-5 and rel_vel < 1e-5


def test_kinematic_limits():
    w = workloads.plain()
    o = oracle.step(w.params, w.pos, w.fwd, w.acc, dt=0.1)
    speed = o["fwd"][:, 3]
    assert np.all(speed <= 1.0 + 1e-6)
    assert np.all((o["pos"][:, :3] >= 0) & (o["pos"][:, :3] < 64.0))
    nrm = np.linalg.norm(o["fwd"][:, :3], axis=1)
    assert np.allclose(nrm, 1.0, atol=1e-5)
    # acceleration change per step bounded by maxForce / mass * smoothRate
    assert np.all(np.linalg.norm(o["acc"][:, :3], axis=1) <= 0.1 * 0.4 + 1e-6)


def test_multi_flock_equals_separate_flocks():
    a = workloads.plain(n=300, L=24.0, M=8, seed=1)
    b = workloads.plain(n=500, L=28.0, M=8, seed=2)
    ob = oracle.step(a.params + b.params, np.concatenate([a.pos, b.pos]), np.concatenate([a.fwd, b.fwd]),
                     np.concatenate([a.acc, b.acc]), dt=0.1)
    oa = oracle.step(a.params, a.pos, a.fwd, a.acc, dt=0.1)
    oc = oracle.step(b.params, b.pos, b.fwd, b.acc, dt=0.1)
    assert np.array_equal(ob["pos"][:300], oa["pos"]) and np.array_equal(ob["pos"][300:], oc["pos"])
    assert np.array_equal(ob["fwd"][300:], oc["fwd"])


@pytest.mark.parametrize("name", sorted(p.stem for p in GOLDEN.glob("oracle_*.npz")))
def test_golden_fixtures(name):
    from tests.golden.make_golden import CASES, run_case
    data = np.load(GOLDEN / (name + ".npz"))
    out = run_case(CASES[name])
    for k in data.files:
        assert np.array_equal(out[k], data[k]), (name, k)


def test_hash_of_non_finite_and_outside_positions():
    """calcGridPos (envgrid3d_resources.cu:60-67) assigns floor(x / cell) to
    an int in device code: the conversion saturates and takes NaN to 0, and
    calcGridHash clamps into the grid.  So +inf and values past the int range
    hash into the last cell, NaN, -inf and negative values into cell 0."""
    w = _small(n=8, L=16.0, M=4, seed=2)
    w.pos[:, :3] = 6.0
    xs = [np.nan, np.inf, -np.inf, 1e30, -5.0, 19.0, -1e30, 15.999]
    want = [0, 3, 0, 3, 0, 3, 0, 3]
    w.pos[:, 0] = np.array(xs, np.float32)
    o = oracle.step(w.params, w.pos, w.fwd, w.acc, dt=0.1)
    key_of_id = np.empty(8, np.int64)
    key_of_id[o["ids"]] = o["keys"]
    home = (1 * 4 + 1) * 4  # y and z in cell 1
    assert key_of_id.tolist() == [home + g for g in want]
