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
        ("lists", _vp), ("steer4", _vp), ("scanned", _vp),
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
        _LIB = L
    return _LIB


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
         threads: int = 0, want_intermediates: bool = True) -> dict:
    """One oracle step.  mode 0: float32 in/out; mode 1: float64 in/out.

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
                  _p(out.get("lists")), _p(out.get("steer")), _p(out.get("scanned")))
    arr = (BrtParams * len(params))(*params)
    if threads <= 0:
        threads = min(hardware_threads(), int(os.environ.get("BRT_ORACLE_THREADS", "64")))
    rc = lib().oracle_step(mode, len(params), C.cast(arr, _vp), float(dt), C.byref(io), threads)
    if rc:
        raise RuntimeError("oracle_step failed: %d" % rc)
    return out
