"""Python mirror of the reference's engine functionalities over the C-ABI.

`Engine` exposes the plugin chain's per-frame methods under the reference's
names (EnvGrid3DPlugIn::reorderSimData, Proximity3DPlugIn::computeNeighborhoods,
OpenSteerWrapperPlugIn::computeSeparations ... applySteeringForces,
BehaviorClusteringPlugIn::steerForClustering) and the getters of the features
they produce (getPos, getForward, getHash, getCellStart, neighbour lists).
Every call goes through libbehavert_b200.so; nothing here computes.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Sequence

import numpy as np

from ._abi import (BRT_MEM_DEVICE, BRT_MEM_HOST, BrtParams, check, lib, ptr)


class Engine:
    """One or many flocks simulated on one GPU (a `brt_engine`)."""

    def __init__(self, flocks: Sequence[BrtParams] | BrtParams, device: int = 0):
        if isinstance(flocks, BrtParams):
            flocks = [flocks]
        arr = (BrtParams * len(flocks))(*flocks)
        h = C.c_void_p()
        check(lib().brt_engine_create(arr, len(flocks), device, C.byref(h)), "brt_engine_create")
        self._h = h
        self.flocks = [f.copy() for f in flocks]
        n = C.c_uint32()
        check(lib().brt_engine_num_agents(h, C.byref(n)), "num_agents")
        self.num_agents = n.value
        check(lib().brt_engine_num_cells(h, C.byref(n)), "num_cells")
        self.num_cells = n.value
        check(lib().brt_neighbor_list_stride(h, C.byref(n)), "list_stride")
        self.list_stride = n.value
        self.features_count = max(int(f.featuresCount) for f in flocks)

    # -- lifetime -------------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_h", None):
            check(lib().brt_engine_destroy(self._h), "brt_engine_destroy")
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    def set_params(self, flock: int, p: BrtParams) -> None:
        check(lib().brt_engine_set_params(self._h, flock, C.byref(p)), "brt_engine_set_params")
        self.flocks[flock] = p.copy()

    def set_option(self, key: str, value: int) -> None:
        check(lib().brt_engine_set_option(self._h, key.encode(), int(value)), "brt_engine_set_option")

    def sync(self) -> None:
        check(lib().brt_sync(self._h), "brt_sync")

    def record_lists(self, enable: bool = True) -> None:
        check(lib().brt_engine_record_lists(self._h, int(enable)), "record_lists")

    def stream_handle(self) -> int:
        s = C.c_void_p()
        check(lib().brt_engine_stream(self._h, C.byref(s)), "brt_engine_stream")
        return s.value or 0

    def device_error(self) -> int:
        w = C.c_uint32()
        check(lib().brt_engine_check_device_error(self._h, C.byref(w)), "check_device_error")
        return w.value

    # -- features ---------------------------------------------------------------
    @staticmethod
    def _where(a) -> int:
        if a is None or isinstance(a, np.ndarray):
            return BRT_MEM_HOST
        return BRT_MEM_DEVICE if getattr(a, "is_cuda", False) else BRT_MEM_HOST

    def set_state(self, pos4=None, fwd4=None, acc4=None, features=None) -> None:
        arrays = [a for a in (pos4, fwd4, acc4, features) if a is not None]
        where = self._where(arrays[0]) if arrays else BRT_MEM_HOST
        check(lib().brt_set_state(self._h, ptr(pos4), ptr(fwd4), ptr(acc4), ptr(features), where), "brt_set_state")

    def get_state(self, features: bool = True):
        n = self.num_agents
        pos = np.empty((n, 4), np.float32)
        fwd = np.empty((n, 4), np.float32)
        acc = np.empty((n, 4), np.float32)
        feat = np.empty((n, self.features_count), np.float32) if (features and self.features_count) else None
        check(lib().brt_get_state(self._h, ptr(pos), ptr(fwd), ptr(acc), ptr(feat), BRT_MEM_HOST), "brt_get_state")
        return pos, fwd, acc, feat

    def get_state_into(self, pos4=None, fwd4=None, acc4=None, features=None) -> None:
        arrays = [a for a in (pos4, fwd4, acc4, features) if a is not None]
        where = self._where(arrays[0]) if arrays else BRT_MEM_HOST
        check(lib().brt_get_state(self._h, ptr(pos4), ptr(fwd4), ptr(acc4), ptr(features), where), "brt_get_state")

    def set_similarity_stats(self, stats4) -> None:
        check(lib().brt_set_similarity_stats(self._h, ptr(stats4), self._where(stats4)), "set_similarity_stats")

    def get_similarity_stats(self) -> np.ndarray:
        out = np.empty((self.num_agents, 4), np.float32)
        check(lib().brt_get_similarity_stats(self._h, ptr(out), BRT_MEM_HOST), "get_similarity_stats")
        return out

    # -- plugin extension: registered per-agent arrays and user kernels ----------------
    def add_array(self, bytes_per_agent: int) -> int:
        """Registers a zero-filled per-agent array that moves with its agents
        (brt_engine_add_array); returns its id."""
        out = C.c_uint32(0)
        check(lib().brt_engine_add_array(self._h, int(bytes_per_agent), C.byref(out)), "brt_engine_add_array")
        return int(out.value)

    def array_set(self, array_id: int, values) -> None:
        """Loads a registered array from agent-id order (a host array, or a
        CUDA tensor)."""
        nbytes = int(self.get_arrays().user_bytes[int(array_id)]) * self.num_agents
        have = values.nbytes if isinstance(values, np.ndarray) else values.numel() * values.element_size()
        if have != nbytes:
            raise ValueError("array %d holds %d bytes, got %d" % (array_id, nbytes, have))
        check(lib().brt_engine_array_set(self._h, int(array_id), ptr(values), self._where(values)),
              "brt_engine_array_set")

    def array_get(self, array_id: int, dtype=np.uint32, shape=None) -> np.ndarray:
        """A registered array in agent-id order."""
        nbytes = int(self.get_arrays().user_bytes[int(array_id)])
        out = np.empty(self.num_agents * nbytes // np.dtype(dtype).itemsize, dtype)
        check(lib().brt_engine_array_get(self._h, int(array_id), ptr(out), BRT_MEM_HOST), "brt_engine_array_get")
        return out.reshape(shape if shape is not None else (self.num_agents, -1))

    def get_arrays(self):
        """The brt_arrays view of the engine's device arrays (raw addresses)."""
        from ._abi import BrtArrays
        view = BrtArrays()
        check(lib().brt_engine_get_arrays(self._h, C.byref(view)), "brt_engine_get_arrays")
        return view

    def launch(self, fn) -> None:
        """Calls fn(stream_handle, view) in stream order (brt_engine_launch);
        fn enqueues its own work on the engine's stream."""
        from ._abi import LAUNCH_FN
        errors = []

        def tramp(_user, stream, view):
            try:
                fn(int(stream or 0), view.contents)
            except Exception as exc:  # re-raised once the C call has returned
                errors.append(exc)

        cb = LAUNCH_FN(tramp)
        check(lib().brt_engine_launch(self._h, cb, None), "brt_engine_launch")
        if errors:
            raise errors[0]

    # -- the fused step ---------------------------------------------------------------
    def step(self, dt: float, nsteps: int = 1) -> None:
        check(lib().brt_step(self._h, dt, nsteps), "brt_step")

    def step_prepare(self, dt: float, nsteps: int) -> None:
        check(lib().brt_step_prepare(self._h, dt, nsteps), "brt_step_prepare")

    def stage_timing(self, enable: bool = True) -> None:
        check(lib().brt_engine_stage_timing(self._h, int(enable)), "brt_engine_stage_timing")

    def stage_times(self):
        """(ms per stage [hash, sort, reorder, fused] summed, timed steps, launches per step)."""
        ms = (C.c_double * 4)()
        steps = C.c_uint64()
        launches = C.c_uint32()
        check(lib().brt_engine_stage_times(self._h, ms, C.byref(steps), C.byref(launches)), "brt_engine_stage_times")
        return list(ms), steps.value, launches.value

    # -- stage-wise functionalities (reference names) --------------------------------------
    def reorderSimData(self) -> None:
        check(lib().brt_reorder_sim_data(self._h), "reorderSimData")

    def computeNeighborhoods(self) -> None:
        check(lib().brt_compute_neighborhoods(self._h), "computeNeighborhoods")

    def resetSteerForce(self) -> None:
        check(lib().brt_reset_steer_force(self._h), "resetSteerForce")

    def computeSeparations(self) -> None:
        check(lib().brt_compute_separations(self._h), "computeSeparations")

    def computeAlignments(self) -> None:
        check(lib().brt_compute_alignments(self._h), "computeAlignments")

    def computeCohesions(self) -> None:
        check(lib().brt_compute_cohesions(self._h), "computeCohesions")

    def steerForClustering(self) -> None:
        check(lib().brt_steer_for_clustering(self._h), "steerForClustering")

    def computeSeekingsWorldCenter(self) -> None:
        check(lib().brt_compute_seekings_world_center(self._h), "computeSeekingsWorldCenter")

    def steerAndSlowToAvoidNeighbors(self) -> None:
        check(lib().brt_steer_and_slow_to_avoid_neighbors(self._h), "steerAndSlowToAvoidNeighbors")

    def applySteeringForces(self, dt: float) -> None:
        check(lib().brt_apply_steering_forces(self._h, dt), "applySteeringForces")

    def steerForMoveAwayBaseTarget(self, base, params=None) -> None:
        """Flee the point `base` (avoidBase); params = avoidBaseParams
        (weight, acceleration factor, radius), None for the defaults."""
        b = np.ascontiguousarray(base, np.float32).reshape(3)
        p = None if params is None else np.ascontiguousarray(params, np.float32).reshape(3)
        check(lib().brt_steer_for_move_away_base_target(self._h, ptr(b), ptr(p)), "steerForMoveAwayBaseTarget")

    def update_crowd(self, dt: float, avoid_base=None, avoid_base_params=None) -> None:
        """The crowd sample's per-frame sequence (Terrain.h:342-366) without
        the terrain plugin: separation replaced by steerAndSlowToAvoidNeighbors,
        and, when avoid_base is given, the move-away-from-base stage after
        cohesion."""
        self.reorderSimData()
        self.computeNeighborhoods()
        self.resetSteerForce()
        self.steerAndSlowToAvoidNeighbors()
        self.computeAlignments()
        self.computeCohesions()
        if avoid_base is not None:
            self.steerForMoveAwayBaseTarget(avoid_base, avoid_base_params)
        self.computeSeekingsWorldCenter()
        self.applySteeringForces(dt)

    def update_stagewise(self, dt: float) -> None:
        """The BehaveRT_Clustering per-frame sequence, stage by stage."""
        self.reorderSimData()
        self.computeNeighborhoods()
        self.resetSteerForce()
        self.computeSeparations()
        self.computeAlignments()
        self.computeCohesions()
        self.steerForClustering()
        self.computeSeekingsWorldCenter()
        self.applySteeringForces(dt)

    # -- getters ------------------------------------------------------------------------------
    def getHash(self):
        n = self.num_agents
        keys = np.empty(n, np.uint32)
        ids = np.empty(n, np.uint32)
        check(lib().brt_get_hash(self._h, ptr(keys), ptr(ids), BRT_MEM_HOST), "getHash")
        return keys, ids

    def getCellRanges(self):
        cs = np.empty(self.num_cells, np.uint32)
        ce = np.empty(self.num_cells, np.uint32)
        check(lib().brt_get_cell_ranges(self._h, ptr(cs), ptr(ce), BRT_MEM_HOST), "getCellStart")
        return cs, ce

    def getNeighborLists(self) -> np.ndarray:
        out = np.empty((self.num_agents, self.list_stride), np.uint32)
        check(lib().brt_get_neighbor_lists(self._h, ptr(out), BRT_MEM_HOST), "neighbor lists")
        return out

    def getSteerForce(self) -> np.ndarray:
        out = np.empty((self.num_agents, 4), np.float32)
        check(lib().brt_get_steer_force(self._h, ptr(out), BRT_MEM_HOST), "getSteerForce")
        return out

    def save_snapshot(self, path) -> None:
        check(lib().brt_save_snapshot(self._h, str(path).encode()), "brt_save_snapshot")

    def load_snapshot(self, path) -> None:
        check(lib().brt_load_snapshot(self._h, str(path).encode()), "brt_load_snapshot")

    # -- BehaviorClustering analytics ------------------------------------------------
    def computeClusterMembership(self, iterations: int = 10) -> None:
        check(lib().brt_compute_cluster_membership(self._h, iterations), "computeClusterMembership")

    def analyzeClusterHitRate(self, same_cluster_max_radius: float = 1.5) -> None:
        check(lib().brt_analyze_cluster_hit_rate(self._h, same_cluster_max_radius), "analyzeClusterHitRate")

    def getClusterMembership(self) -> np.ndarray:
        out = np.empty((self.num_agents, 4), np.float32)
        check(lib().brt_get_cluster_membership(self._h, ptr(out), BRT_MEM_HOST), "getClusterMembership")
        return out

    def autotune(self, dt: float, steps: int = 10) -> dict:
        """Times launch configurations on the current state, keeps the
        fastest and returns the choice with every trial's ms per step."""
        import json
        buf = C.create_string_buffer(8192)
        check(lib().brt_engine_autotune(self._h, dt, steps, buf, len(buf)), "brt_engine_autotune")
        return json.loads(buf.value.decode())

    # -- differentiable rollout (no reference counterpart) -----------------------
    def set_steering_weights(self, weights) -> None:
        """Per-flock (separation, alignment, cohesion) weights, nflocks x 3."""
        if isinstance(weights, np.ndarray) or not getattr(weights, "is_cuda", False):
            weights = np.ascontiguousarray(np.asarray(weights, np.float32).reshape(-1, 3))
        check(lib().brt_set_steering_weights(self._h, ptr(weights), self._where(weights)), "set_steering_weights")

    def get_steering_weights(self) -> np.ndarray:
        out = np.empty((len(self.flocks), 3), np.float32)
        check(lib().brt_get_steering_weights(self._h, ptr(out), BRT_MEM_HOST), "get_steering_weights")
        return out

    def adjoint_forward(self, target_pos4, nsteps: int, checkpoint_every: int, dt: float) -> np.ndarray:
        """Taped forward of nsteps steps; returns the FP64 loss of every flock
        (mean squared minimum-image distance of final positions to targets)."""
        if isinstance(target_pos4, np.ndarray):
            t = np.zeros((self.num_agents, 4), np.float32)
            t[:, :target_pos4.shape[1]] = target_pos4[:, :4]
            target_pos4 = t
        loss = np.empty(len(self.flocks), np.float64)
        check(lib().brt_adjoint_forward(self._h, dt, nsteps, checkpoint_every, ptr(target_pos4),
                                        self._where(target_pos4), ptr(loss)), "brt_adjoint_forward")
        return loss

    def adjoint_backward(self, loss_scale=None, gpos_T=None, gfwd_T=None, gacc_T=None) -> dict:
        """Gradients of sum_f loss_scale[f] * loss_f (+ <g_T, final state>)
        with respect to the initial state and the per-flock weights."""
        n = self.num_agents
        scale = None if loss_scale is None else np.ascontiguousarray(loss_scale, np.float64)
        extras = []
        for g in (gpos_T, gfwd_T, gacc_T):
            if g is None:
                extras.append(None)
            else:
                e = np.zeros((n, 4), np.float32)
                e[:, :g.shape[1]] = g
                extras.append(e)
        out = {k: np.empty((n, 4), np.float32) for k in ("pos", "fwd", "vel", "acc")}
        out["weights"] = np.empty((len(self.flocks), 3), np.float64)
        check(lib().brt_adjoint_backward(self._h, ptr(scale), ptr(extras[0]), ptr(extras[1]), ptr(extras[2]),
                                         BRT_MEM_HOST, ptr(out["pos"]), ptr(out["fwd"]), ptr(out["vel"]),
                                         ptr(out["acc"]), ptr(out["weights"]), BRT_MEM_HOST), "brt_adjoint_backward")
        return out

    def adjoint_tape(self, nsteps: int):
        """Frozen lists (T x N x stride, neighbour agent ids) and flag words
        (T x N x 4) of the last backward (needs option adjoint_export)."""
        lists = np.empty((nsteps, self.num_agents, self.list_stride), np.uint32)
        flags = np.empty((nsteps, self.num_agents, 4), np.uint32)
        check(lib().brt_adjoint_get_tape(self._h, ptr(lists), ptr(flags), BRT_MEM_HOST), "brt_adjoint_get_tape")
        return lists, flags

    def adjoint_tape_states(self, nsteps: int):
        """Input state of every step of the last backward (T x N x 4 each:
        position, forward with speed in w, smoothed acceleration; by agent id;
        needs option adjoint_export)."""
        out = [np.empty((nsteps, self.num_agents, 4), np.float32) for _ in range(3)]
        check(lib().brt_adjoint_get_tape_states(self._h, *(ptr(x) for x in out), BRT_MEM_HOST),
              "brt_adjoint_get_tape_states")
        return tuple(out)


def radix_sort_pairs(pairs_in, pairs_out, n: int, bits: int, scratch, stream: Optional[int] = None) -> None:
    """Standalone onesweep sort of uint2 (key, value) pairs on device memory."""
    nbytes = scratch.numel() * scratch.element_size() if hasattr(scratch, "numel") else scratch.nbytes
    check(lib().brt_radix_sort_pairs(ptr(pairs_in), ptr(pairs_out), n, bits, ptr(scratch), nbytes,
                                     C.c_void_p(stream) if stream else None), "brt_radix_sort_pairs")


def radix_sort_scratch_bytes(n: int, bits: int) -> int:
    return int(lib().brt_radix_sort_scratch_bytes(n, bits))
