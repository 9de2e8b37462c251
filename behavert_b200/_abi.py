"""ctypes mirror of include/behavert_b200.h and the loader of the CUDA library.

The library is loaded from this package directory only.  There is no CPU
fallback: if libbehavert_b200.so is missing, importing the engine API raises.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

BRT_OK = 0
BRT_ERR_CUDA = 1
BRT_ERR_CONFIG = 2
BRT_ERR_CAPACITY = 3
BRT_ERR_TIMEOUT = 4
BRT_ERR_ARG = 5
BRT_ERR_STATE = 6
BRT_ERR_NODEVICE = 7
BRT_MEM_HOST = 0
BRT_MEM_DEVICE = 1
BRT_MAX_NEIGHBORS = 128
BRT_MAX_FEATUREDIM = 32
BRT_MAX_OBSTACLES = 64

F3 = C.c_float * 3


class SchoolingParams(C.Structure):
    """Mirror of struct brt_schooling_params (SchoolingParams field names)."""

    _fields_ = [
        ("mode", C.c_int32),
        ("theta", C.c_float),
        ("delta", C.c_float),
        ("r_r", C.c_float),
        ("r_p", C.c_float),
        ("eta", C.c_float),
        ("w_a", C.c_float),
        ("w_o", C.c_float),
        ("s", C.c_float),
        ("randomDeviationWeight", C.c_float),
        ("seed", C.c_uint32),
    ]


class BrtParams(C.Structure):
    """Mirror of brt_params (field names of the reference's parameter structs)."""

    _fields_ = [
        ("numBodies", C.c_uint32),
        ("commonRadius", C.c_float),
        ("use2DProjection", C.c_int32),
        ("worldSize", C.c_float),
        ("cellSize", C.c_float),
        ("maxBodiesPerCell", C.c_uint32),
        ("disableSorting", C.c_int32),
        ("maxNeighbors", C.c_uint32),
        ("useKnn", C.c_int32),
        ("commonSearchRadius", C.c_float),
        ("commonMaxSpeed", C.c_float),
        ("commonMaxForce", C.c_float),
        ("commonMass", C.c_float),
        ("commonSensingMinRadius", C.c_float),
        ("separationParams", F3),
        ("cohesionParams", F3),
        ("alignmentParams", F3),
        ("featuresCount", C.c_uint32),
        ("clusteringForceParams", F3),
        ("alignmentClusteringForceParams", F3),
        ("similarityStatsParams", F3),
        ("avgSimilarityController", C.c_float),
        ("featureRelaxRate", C.c_float),
        ("numObstacles", C.c_uint32),
        ("obstacleAvoidanceWeight", C.c_float),
        ("obstacles", (C.c_float * 4) * BRT_MAX_OBSTACLES),
        ("schooling", SchoolingParams),
    ]

    def set_obstacles(self, arr) -> None:
        arr = np.asarray(arr, dtype=np.float32).reshape(-1, 4)
        if len(arr) > BRT_MAX_OBSTACLES:
            raise ValueError("at most %d obstacles per flock" % BRT_MAX_OBSTACLES)
        self.numObstacles = len(arr)
        for k, row in enumerate(arr):
            for a in range(4):
                self.obstacles[k][a] = float(row[a])

    def copy(self) -> "BrtParams":
        p = BrtParams()
        C.pointer(p)[0] = self
        return p


_LIB = None
LIB_PATH = Path(__file__).resolve().parent / "libbehavert_b200.so"

_vp = C.c_void_p
_u32p = C.POINTER(C.c_uint32)
_fp = C.POINTER(C.c_float)

MAX_USER_ARRAYS = 8


class BrtArrays(C.Structure):
    """brt_arrays: a view of the engine's device arrays (raw addresses)."""
    _fields_ = [
        ("num_agents", C.c_uint32), ("num_cells", C.c_uint32), ("features_stride", C.c_uint32),
        ("list_stride", C.c_uint32),
        ("pos4", _vp), ("forward4", _vp), ("smooth_accel4", _vp), ("features", _vp), ("agent_id", _vp),
        ("sorted_pos4", _vp), ("sorted_forward4", _vp), ("sorted_smooth_accel4", _vp), ("sorted_features", _vp),
        ("sorted_agent_id", _vp), ("steer4", _vp), ("neighbor_lists", _vp), ("cell_start", _vp), ("cell_end", _vp),
        ("num_user", C.c_uint32), ("user_bytes", C.c_uint32 * MAX_USER_ARRAYS), ("user", _vp * MAX_USER_ARRAYS),
        ("user_agent_id", _vp),
    ]


LAUNCH_FN = C.CFUNCTYPE(None, _vp, _vp, C.POINTER(BrtArrays))

_SIGS = {
    "brt_version": (C.c_char_p, []),
    "brt_error_string": (C.c_char_p, [C.c_int]),
    "brt_last_error": (C.c_char_p, []),
    "brt_device_count": (C.c_int, [C.POINTER(C.c_int)]),
    "brt_params_default": (C.c_int, [C.POINTER(BrtParams)]),
    "brt_engine_create": (C.c_int, [C.POINTER(BrtParams), C.c_uint32, C.c_int, C.POINTER(_vp)]),
    "brt_engine_destroy": (C.c_int, [_vp]),
    "brt_engine_num_agents": (C.c_int, [_vp, _u32p]),
    "brt_engine_num_cells": (C.c_int, [_vp, _u32p]),
    "brt_engine_set_params": (C.c_int, [_vp, C.c_uint32, C.POINTER(BrtParams)]),
    "brt_engine_set_option": (C.c_int, [_vp, C.c_char_p, C.c_int64]),
    "brt_engine_stream": (C.c_int, [_vp, C.POINTER(_vp)]),
    "brt_sync": (C.c_int, [_vp]),
    "brt_set_state": (C.c_int, [_vp, _vp, _vp, _vp, _vp, C.c_int]),
    "brt_get_state": (C.c_int, [_vp, _vp, _vp, _vp, _vp, C.c_int]),
    "brt_set_similarity_stats": (C.c_int, [_vp, _vp, C.c_int]),
    "brt_get_similarity_stats": (C.c_int, [_vp, _vp, C.c_int]),
    "brt_step": (C.c_int, [_vp, C.c_float, C.c_uint32]),
    "brt_step_prepare": (C.c_int, [_vp, C.c_float, C.c_uint32]),
    "brt_engine_stage_timing": (C.c_int, [_vp, C.c_int]),
    "brt_engine_stage_times": (C.c_int, [_vp, C.POINTER(C.c_double), C.POINTER(C.c_uint64), _u32p]),
    "brt_reorder_sim_data": (C.c_int, [_vp]),
    "brt_compute_neighborhoods": (C.c_int, [_vp]),
    "brt_reset_steer_force": (C.c_int, [_vp]),
    "brt_compute_separations": (C.c_int, [_vp]),
    "brt_compute_alignments": (C.c_int, [_vp]),
    "brt_compute_cohesions": (C.c_int, [_vp]),
    "brt_steer_for_clustering": (C.c_int, [_vp]),
    "brt_compute_seekings_world_center": (C.c_int, [_vp]),
    "brt_steer_and_slow_to_avoid_neighbors": (C.c_int, [_vp]),
    "brt_steer_for_move_away_base_target": (C.c_int, [_vp, _vp, _vp]),
    "brt_engine_add_array": (C.c_int, [_vp, C.c_uint32, _u32p]),
    "brt_engine_array_set": (C.c_int, [_vp, C.c_uint32, _vp, C.c_int]),
    "brt_engine_array_get": (C.c_int, [_vp, C.c_uint32, _vp, C.c_int]),
    "brt_engine_get_arrays": (C.c_int, [_vp, C.POINTER(BrtArrays)]),
    "brt_engine_launch": (C.c_int, [_vp, LAUNCH_FN, _vp]),
    "brt_apply_steering_forces": (C.c_int, [_vp, C.c_float]),
    "brt_get_hash": (C.c_int, [_vp, _vp, _vp, C.c_int]),
    "brt_get_cell_ranges": (C.c_int, [_vp, _vp, _vp, C.c_int]),
    "brt_get_neighbor_lists": (C.c_int, [_vp, _vp, C.c_int]),
    "brt_neighbor_list_stride": (C.c_int, [_vp, _u32p]),
    "brt_get_steer_force": (C.c_int, [_vp, _vp, C.c_int]),
    "brt_engine_record_lists": (C.c_int, [_vp, C.c_int]),
    "brt_engine_check_device_error": (C.c_int, [_vp, _u32p]),
    "brt_save_snapshot": (C.c_int, [_vp, C.c_char_p]),
    "brt_load_snapshot": (C.c_int, [_vp, C.c_char_p]),
    "brt_compute_cluster_membership": (C.c_int, [_vp, C.c_uint32]),
    "brt_analyze_cluster_hit_rate": (C.c_int, [_vp, C.c_float]),
    "brt_get_cluster_membership": (C.c_int, [_vp, _vp, C.c_int]),
    "brt_school_repulsion": (C.c_int, [_vp]),
    "brt_school_attraction_orientation": (C.c_int, [_vp]),
    "brt_school_movement": (C.c_int, [_vp]),
    "brt_school_animate": (C.c_int, [_vp]),
    "brt_engine_autotune": (C.c_int, [_vp, C.c_float, C.c_uint32, C.c_char_p, C.c_size_t]),
    "brt_adjoint_forward": (C.c_int, [_vp, C.c_float, C.c_uint32, C.c_uint32, _vp, C.c_int, _vp]),
    "brt_adjoint_backward": (C.c_int, [_vp, _vp, _vp, _vp, _vp, C.c_int, _vp, _vp, _vp, _vp, _vp, C.c_int]),
    "brt_adjoint_get_tape": (C.c_int, [_vp, _vp, _vp, C.c_int]),
    "brt_adjoint_get_tape_states": (C.c_int, [_vp, _vp, _vp, _vp, C.c_int]),
    "brt_set_steering_weights": (C.c_int, [_vp, _vp, C.c_int]),
    "brt_get_steering_weights": (C.c_int, [_vp, _vp, C.c_int]),
    "brt_radix_sort_scratch_bytes": (C.c_size_t, [C.c_uint32, C.c_uint32]),
    "brt_radix_sort_pairs": (C.c_int, [_vp, _vp, C.c_uint32, C.c_uint32, _vp, C.c_size_t, _vp]),
    "brt_radix_sort_noalloc_max_pairs": (C.c_size_t, []),
    "brt_radix_sort_pairs_noalloc": (C.c_int, [_vp, _vp, C.c_uint32, C.c_uint32, _vp]),
}

# Every symbol the public header declares (checked by the CPU tests).
EXPORTED_SYMBOLS = tuple(_SIGS.keys())


class BrtError(RuntimeError):
    def __init__(self, status: int, where: str, msg: str):
        super().__init__("%s failed: status %d (%s)" % (where, status, msg))
        self.status = status


def lib():
    """The loaded CUDA library (raises if it was not built)."""
    global _LIB
    if _LIB is None:
        if not LIB_PATH.exists():
            raise RuntimeError(
                "libbehavert_b200.so is not built (run `python -m behavert_b200.build`); "
                "there is no CPU fallback")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = L
    return _LIB


def check(status: int, where: str) -> None:
    if status != BRT_OK:
        msg = lib().brt_last_error().decode(errors="replace")
        raise BrtError(status, where, msg)


def params_default() -> BrtParams:
    p = BrtParams()
    check(lib().brt_params_default(C.byref(p)), "brt_params_default")
    return p


def ptr(a) -> C.c_void_p:
    """Address of a numpy array or a torch tensor (host or device)."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        if not a.flags["C_CONTIGUOUS"]:
            raise ValueError("array must be C-contiguous")
        return C.c_void_p(a.ctypes.data)
    if hasattr(a, "data_ptr"):
        if not a.is_contiguous():
            raise ValueError("tensor must be contiguous")
        return C.c_void_p(a.data_ptr())
    raise TypeError("unsupported buffer type %r" % type(a))
