"""ctypes binding of the CPU oracle (oracle/brt_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline / reference legs of bench.py, never by the product library.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path
from typing import Sequence

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "liboracle_brt.so"

_vp = C.c_void_p
_u32p = C.POINTER(C.c_uint32)


class OracleIO(C.Structure):
    _fields_ = [
        ("pos4", _vp), ("fwd4", _vp), ("acc4", _vp), ("feat", _vp), ("stats4", _vp),
        ("pos4_out", _vp), ("fwd4_out", _vp), ("acc4_out", _vp), ("feat_out", _vp), ("stats4_out", _vp),
        ("sorted_keys", _vp), ("sorted_ids", _vp), ("cell_start", _vp), ("cell_end", _vp),
        ("lists", _vp), ("steer4", _vp), ("scanned", _vp), ("random_step", C.c_uint32),
        ("avoid_neighbors", C.c_uint32), ("move_away", C.c_uint32),
        ("avoid_base", C.c_float * 3), ("avoid_base_params", C.c_float * 3),
    ]


_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        if not LIB_PATH.exists():
            import subprocess
            subprocess.run(["make", "-C", str(HERE)], check=True, capture_output=True)
        from behavert_b200._abi import BrtParams  # noqa: F401  (struct layout shared with the product header)
        L = C.CDLL(str(LIB_PATH))
        L.oracle_step.restype = C.c_int
        L.oracle_step.argtypes = [C.c_int, C.c_uint32, _vp, C.c_float, C.POINTER(OracleIO), C.c_int]
        L.oracle_num_cells.restype = C.c_int
        L.oracle_num_cells.argtypes = [C.c_uint32, _vp, _u32p]
        L.oracle_hardware_threads.restype = C.c_int
        L.oracle_params_default.restype = C.c_int
        L.oracle_params_default.argtypes = [_vp]
        L.oracle_frozen_forward.restype = C.c_int
        L.oracle_frozen_forward.argtypes = [C.c_uint32, _vp, _vp, C.c_uint32, C.c_double, _vp, _vp, _vp, _vp,
                                            _vp, _vp, _vp, _vp, _vp, C.c_int]
        L.oracle_frozen_reverse.restype = C.c_int
        L.oracle_frozen_reverse.argtypes = [C.c_uint32, _vp, _vp, C.c_uint32, C.c_double, _vp, _vp, _vp, _vp,
                                            _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, C.c_int]
        L.oracle_frozen_reverse_at.restype = C.c_int
        L.oracle_frozen_reverse_at.argtypes = [C.c_uint32, _vp, _vp, C.c_uint32, C.c_double, _vp, _vp, _vp, _vp,
                                               _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]
        _LIB = L
    return _LIB


def params_default():
    """BrtParams filled with the workloads' defaults by the oracle library
    (equal, byte for byte, to the CUDA library's brt_params_default), so a
    CPU-only run builds its workload without loading the CUDA library."""
    from behavert_b200._abi import BrtParams
    p = BrtParams()
    rc = lib().oracle_params_default(C.byref(p))
    if rc:
        raise RuntimeError("oracle_params_default failed: %d" % rc)
    return p


def hardware_threads() -> int:
    return int(lib().oracle_hardware_threads())


def _p(a):
    return None if a is None else C.c_void_p(a.ctypes.data)


def num_cells(params: Sequence) -> int:
    from behavert_b200._abi import BrtParams
    arr = (BrtParams * len(params))(*params)
    out = C.c_uint32()
    rc = lib().oracle_num_cells(len(params), C.cast(arr, _vp), C.byref(out))
    if rc:
        raise RuntimeError("oracle_num_cells failed: %d" % rc)
    return out.value


def step(params: Sequence, pos, fwd, acc, feat=None, stats=None, dt: float = 0.1, mode: int = 0,
         threads: int = 0, want_intermediates: bool = True, random_step: int = 0,
         avoid_neighbors: bool = False, move_away=None) -> dict:
    """One oracle step.  mode 0: float32 in/out; mode 1: float64 in/out.
    random_step: the step of the Schooling random stream (schooling.mode 2).
    avoid_neighbors: the crowd sample's order (Terrain.h:342-366), with
    steerAndSlowToAvoidNeighbors in place of computeSeparations.
    move_away: (base xyz, (weight, acceleration factor, radius)) for the
    steerForMoveAwayBaseTarget stage after cohesion, or None.

    Returns the id-ordered new state and, when asked, the sorted keys/ids,
    cell ranges, neighbour lists (stride Mmax+1) and the steering force per
    sorted slot.
    """
    from behavert_b200._abi import BrtParams
    dtype = np.float32 if mode == 0 else np.float64
    n = pos.shape[0]
    Fm = max(int(p.featuresCount) for p in params)
    Mm = max(int(p.maxNeighbors) for p in params)
    C_ = num_cells(params)
    pos = np.ascontiguousarray(pos, dtype)
    fwd = np.ascontiguousarray(fwd, dtype)
    acc = np.ascontiguousarray(acc, dtype)
    feat = np.ascontiguousarray(feat, dtype) if (feat is not None and Fm) else None
    stats = np.ascontiguousarray(stats, dtype) if stats is not None else None
    out = {
        "pos": np.empty((n, 4), dtype), "fwd": np.empty((n, 4), dtype), "acc": np.empty((n, 4), dtype),
        "feat": np.empty((n, Fm), dtype) if Fm else None, "stats": np.empty((n, 4), dtype),
    }
    if want_intermediates:
        out.update({
            "keys": np.empty(n, np.uint32), "ids": np.empty(n, np.uint32),
            "cell_start": np.empty(C_, np.uint32), "cell_end": np.empty(C_, np.uint32),
            "lists": np.zeros((n, Mm + 1), np.uint32), "steer": np.empty((n, 4), dtype),
            "scanned": np.empty(n, np.uint32),
        })
    io = OracleIO(_p(pos), _p(fwd), _p(acc), _p(feat), _p(stats),
                  _p(out["pos"]), _p(out["fwd"]), _p(out["acc"]), _p(out["feat"]), _p(out["stats"]),
                  _p(out.get("keys")), _p(out.get("ids")), _p(out.get("cell_start")), _p(out.get("cell_end")),
                  _p(out.get("lists")), _p(out.get("steer")), _p(out.get("scanned")), int(random_step),
                  int(bool(avoid_neighbors)), int(move_away is not None),
                  (C.c_float * 3)(*([0.0] * 3 if move_away is None else [float(x) for x in move_away[0]])),
                  (C.c_float * 3)(*([0.0] * 3 if move_away is None else [float(x) for x in move_away[1]])))
    arr = (BrtParams * len(params))(*params)
    if threads <= 0:
        threads = min(hardware_threads(), int(os.environ.get("BRT_ORACLE_THREADS", "64")))
    rc = lib().oracle_step(mode, len(params), C.cast(arr, _vp), float(dt), C.byref(io), threads)
    if rc:
        raise RuntimeError("oracle_step failed: %d" % rc)
    return out


# ---------------------------------------------------------------------------
# FP64 frozen-neighbour / frozen-branch model (oracle/brt_oracle_adjoint.cpp)

def _threads(threads: int) -> int:
    if threads <= 0:
        threads = min(hardware_threads(), int(os.environ.get("BRT_ORACLE_THREADS", "64")))
    return threads


def lists_by_id(step_out: dict) -> np.ndarray:
    """Neighbour lists of one oracle step re-indexed by agent id: row id is
    the count, then the neighbours' agent ids in list order."""
    ids = step_out["ids"]
    lists = step_out["lists"]
    out = np.zeros_like(lists)
    n = lists[:, 0]
    out[ids, 0] = n
    stride = lists.shape[1]
    k = np.arange(stride - 1)[None, :]
    valid = k < n[:, None]
    nb = np.where(valid, ids[np.minimum(lists[:, 1:], len(ids) - 1)], 0)
    out[ids, 1:] = nb
    return out


def frozen_forward(params: Sequence, pos, fwd, acc, lists, weights=None, flags=None, dt: float = 0.1,
                   want_flags: bool = False, threads: int = 0) -> dict:
    """FP64 trajectory over len(lists) steps with the given per-step lists
    (T x N x stride, by agent id) and, optionally, frozen branch flags
    (T x N x 4).  Returns the final state (float64, agent-id order)."""
    from behavert_b200._abi import BrtParams
    lists = np.ascontiguousarray(lists, np.uint32)
    T, n = lists.shape[0], lists.shape[1]
    pos = np.ascontiguousarray(pos, np.float64)
    fwd = np.ascontiguousarray(fwd, np.float64)
    acc = np.ascontiguousarray(acc, np.float64)
    w = None if weights is None else np.ascontiguousarray(weights, np.float64).reshape(-1)
    fz = None if flags is None else np.ascontiguousarray(flags, np.uint32)
    fo = np.zeros((T, n, 4), np.uint32) if want_flags else None
    out = {"pos": np.empty((n, 4)), "fwd": np.empty((n, 4)), "acc": np.empty((n, 4))}
    arr = (BrtParams * len(params))(*params)
    rc = lib().oracle_frozen_forward(len(params), C.cast(arr, _vp), _p(w), T, float(dt), _p(pos), _p(fwd), _p(acc),
                                     _p(lists), _p(fz), _p(fo), _p(out["pos"]), _p(out["fwd"]), _p(out["acc"]),
                                     _threads(threads))
    if rc:
        raise RuntimeError("oracle_frozen_forward failed: %d" % rc)
    if want_flags:
        out["flags"] = fo
    return out


def frozen_reverse(params: Sequence, pos, fwd, acc, lists, gpos_T, gfwd_T=None, gacc_T=None, weights=None,
                   flags=None, dt: float = 0.1, threads: int = 0) -> dict:
    """Reverse mode of frozen_forward: adjoint of the initial state and of
    the per-flock weights (nflocks x 3) given the final state's adjoint."""
    from behavert_b200._abi import BrtParams
    lists = np.ascontiguousarray(lists, np.uint32)
    T, n = lists.shape[0], lists.shape[1]
    z = np.zeros((n, 4))
    pos = np.ascontiguousarray(pos, np.float64)
    fwd = np.ascontiguousarray(fwd, np.float64)
    acc = np.ascontiguousarray(acc, np.float64)
    gp = np.ascontiguousarray(gpos_T, np.float64)
    gf = z if gfwd_T is None else np.ascontiguousarray(gfwd_T, np.float64)
    ga = z if gacc_T is None else np.ascontiguousarray(gacc_T, np.float64)
    w = None if weights is None else np.ascontiguousarray(weights, np.float64).reshape(-1)
    fz = None if flags is None else np.ascontiguousarray(flags, np.uint32)
    out = {"pos": np.empty((n, 4)), "fwd": np.empty((n, 4)), "acc": np.empty((n, 4)),
           "weights": np.empty((len(params), 3))}
    arr = (BrtParams * len(params))(*params)
    rc = lib().oracle_frozen_reverse(len(params), C.cast(arr, _vp), _p(w), T, float(dt), _p(pos), _p(fwd), _p(acc),
                                     _p(lists), _p(fz), _p(gp), _p(gf), _p(ga), _p(out["pos"]), _p(out["fwd"]),
                                     _p(out["acc"]), _p(out["weights"]), _threads(threads))
    if rc:
        raise RuntimeError("oracle_frozen_reverse failed: %d" % rc)
    return out


def frozen_reverse_at(params: Sequence, states, lists, gpos_T, gfwd_T=None, gacc_T=None, weights=None,
                      flags=None, dt: float = 0.1) -> dict:
    """frozen_reverse linearised at a given trajectory: states = (pos, fwd,
    acc), each T x N x 4 (the input state of every step, by agent id)."""
    from behavert_b200._abi import BrtParams
    lists = np.ascontiguousarray(lists, np.uint32)
    T, n = lists.shape[0], lists.shape[1]
    pos_t, fwd_t, acc_t = (np.ascontiguousarray(x, np.float64).reshape(T, n, 4) for x in states)
    z = np.zeros((n, 4))
    gp = np.ascontiguousarray(gpos_T, np.float64)
    gf = z if gfwd_T is None else np.ascontiguousarray(gfwd_T, np.float64)
    ga = z if gacc_T is None else np.ascontiguousarray(gacc_T, np.float64)
    w = None if weights is None else np.ascontiguousarray(weights, np.float64).reshape(-1)
    fz = None if flags is None else np.ascontiguousarray(flags, np.uint32)
    out = {"pos": np.empty((n, 4)), "fwd": np.empty((n, 4)), "acc": np.empty((n, 4)),
           "weights": np.empty((len(params), 3))}
    arr = (BrtParams * len(params))(*params)
    rc = lib().oracle_frozen_reverse_at(len(params), C.cast(arr, _vp), _p(w), T, float(dt), _p(pos_t), _p(fwd_t),
                                        _p(acc_t), _p(lists), _p(fz), _p(gp), _p(gf), _p(ga), _p(out["pos"]),
                                        _p(out["fwd"]), _p(out["acc"]), _p(out["weights"]))
    if rc:
        raise RuntimeError("oracle_frozen_reverse_at failed: %d" % rc)
    return out


def min_image(d, L):
    """Minimum image of offsets in a periodic cube of side L."""
    return d - L * np.round(d / L)


# ---------------------------------------------------------------------------
# BehaviorClustering analytics (BehaviorClusteringPlugIn.h:828-894, kernels
# BehaviorClustering_kernel.cu:502-652) over the lists of one step.

def cluster_membership(step_out: dict, iterations: int) -> np.ndarray:
    """Local label propagation: labels (float32, by agent id) start as each
    agent's sorted slot; each sweep takes the minimum over the agent and its
    listed neighbours (all reading the previous sweep)."""
    ids = step_out["ids"]
    lists = step_out["lists"]
    n = len(ids)
    lab = np.empty(n, np.float32)
    lab[ids] = np.arange(n, dtype=np.float32)
    cnt = lists[:, 0]
    valid = np.arange(lists.shape[1] - 1)[None, :] < cnt[:, None]
    nb = ids[np.where(valid, lists[:, 1:], 0)]
    for _ in range(iterations):
        cand = np.where(valid, lab[nb], np.float32(np.inf)).min(axis=1) if valid.shape[1] else np.full(n, np.inf)
        new = np.empty_like(lab)
        new[ids] = np.minimum(lab[ids], cand.astype(np.float32))
        lab = new
    return lab


def cluster_hit_rate(params: Sequence, pos_in, step_out: dict, labels, radius: float) -> np.ndarray:
    """(label, hit rate, mean close-neighbour label) per agent id: among the
    listed neighbours closer than `radius` (float32 distance to the neighbour's
    periodic image), the fraction sharing the label and their mean label, -1
    without any; sums in list order in float32."""
    ids = step_out["ids"]
    lists = step_out["lists"]
    n = len(ids)
    L = np.float32(params[0].worldSize)
    cell = np.float32(params[0].cellSize)
    G = int(round(float(L) / float(cell)))
    ps = np.ascontiguousarray(pos_in, np.float32)[ids, :3]

    def grid(x):
        # the device's float-to-int conversion takes NaN to 0 and saturates
        return np.nan_to_num(np.clip(np.floor(x / cell), 0, G - 1), nan=0.0).astype(np.int64)

    gi = grid(ps)
    my = labels[ids]
    close = np.zeros(n, np.int64)
    real = np.zeros(n, np.float32)
    hit = np.zeros(n, np.float32)
    cnt = lists[:, 0]
    for k in range(lists.shape[1] - 1):
        valid = k < cnt
        j = np.where(valid, lists[:, 1 + k], 0)
        q = ps[j].copy()
        gj = grid(q)
        shift = np.where((gi == 0) & (gj == G - 1), -L, np.where((gi == G - 1) & (gj == 0), L, np.float32(0)))
        q = (q + shift.astype(np.float32)).astype(np.float32)
        d = (q - ps).astype(np.float32)
        dist = np.sqrt(((d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2]).astype(np.float32))
        use = valid & ~(dist > np.float32(radius))
        other = labels[ids[j]]
        close += use
        real = np.where(use, (real + other).astype(np.float32), real)
        hit = np.where(use & (my == other), (hit + np.float32(1)).astype(np.float32), hit)
    out = np.zeros((n, 4), np.float32)
    c = close.astype(np.float32)
    hr = np.where(close > 0, hit / np.where(close > 0, c, 1), hit).astype(np.float32)
    rl = np.where(close > 0, real / np.where(close > 0, c, 1), np.float32(-1)).astype(np.float32)
    out[ids, 0] = my
    out[ids, 1] = hr
    out[ids, 2] = rl
    return out
