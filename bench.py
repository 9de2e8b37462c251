#!/usr/bin/env python
"""Benchmark of the per-step agent pipeline (config 1: 1,048,576 agents).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One "step" is one simulation step of the whole flock: cell hash, onesweep
sort, reorder + cell ranges, fused neighbour search / steering / integration /
feature relaxation.  Rank 0 prints one JSON line.

* value: agent-steps/s with the state resident in HBM, K steps launched as one
  CUDA graph, timed with CUDA events on the engine stream (max over ranks).
* e2e: the same metric through the public C-ABI with host buffers: every e2e
  iteration uploads the state from pinned host memory (brt_set_state), runs the
  config's 100-step horizon (brt_step) and reads the state back
  (brt_get_state); the copies are inside the timed region.
* roofline: the dominant kernel (fused pass) against the measured HBM copy
  bandwidth, with per-stage CUDA-event times from a second timed pass.
* cpu_baseline (rank 0, N=1): the CPU oracle (multi-threaded C++ restatement of
  the reference's plugin logic) on a bounded sample of the same workload, plus
  the per-step error of the GPU state against the FP64 oracle.
* batched / adjoint / fitting (N=1): configs 2, 3 and 4.
* next_rows (rank 0, N=1): the components beside the flocking path (Schooling,
  kNN lists, the crowd order with steerAndSlowToAvoidNeighbors, clustering
  analytics, snapshots) on 1,048,576-agent states, each with the oracle's
  host time for the same work and a parity check of its first step.

Multi-GPU: the path does not shard (one flock on one GPU); N ranks run N
independent replicas ("weak" scaling), one process per GPU.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "agent-steps/s (1M agents, 1 B200)"
UNIT = "agent-steps/s"
WORKLOAD = ("config 1: plain large flocking, 1,048,576 agents (70% uniform, 30% in 64 Gaussian blobs sigma 6), "
            "periodic cube 256, cell 4, radius 4, maxNeighbors 32, weights 1.5/1/1, 8 features relaxed at 0.05, "
            "dt 0.1, FP32")
E2E_HORIZON = 100  # config 1 runs 100 steps


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def alg_bytes_per_agent_step(num_cells: int, n: int, features: int, passes_8bit: int) -> dict:
    """Algorithmic HBM bytes per agent-step (plain): 40 + 16P + 4S per agent,
    S = 48 + 4F, P = 8-bit sort passes, plus 8 bytes per cell per step."""
    S = 48 + 4 * features
    per_agent = 40 + 16 * passes_8bit + 4 * S
    fused = 4 + 2 * S
    return {"per_agent_step": per_agent + 8.0 * num_cells / n, "fused_per_agent": fused, "S": S}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.time(), line.strip()))

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self, t0, t1):
        rows = []
        for t, line in self.lines:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            rows.append((t, parts))
        inside = [r for t, r in rows if t0 - 0.15 <= t <= t1 + 0.15] or [r for _, r in rows]
        if not inside:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        sm = [float(r[1]) for r in inside if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in inside if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in inside for k in range(4) if r[5 + k].strip() == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(inside)}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def max_over_ranks(pg, ms: float, device) -> float:
    """The largest of the ranks' device times (one all-reduce; every rank
    calls it at the same point, and a single process returns its own)."""
    if pg is None:
        return ms
    import torch
    t = torch.tensor([ms], device=device, dtype=torch.float64)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def replica_value(world: int, agents: int, steps: int, ms: float) -> float:
    """Whole-job agent-steps/s of `world` replicas of `agents` agents each,
    every one stepping `steps` steps, the job taking the slowest rank's `ms`."""
    return world * agents * steps / (ms / 1e3)


def _horizons(steps: int, horizon: int = E2E_HORIZON):
    """Split `steps` into runs of at most `horizon` steps, each restarting from
    the seeded state (config 1 is a 100-step run from its seeded state)."""
    out = []
    while steps > 0:
        out.append(min(horizon, steps))
        steps -= out[-1]
    return out


def bench_config(world: int) -> dict:
    """The workload description; both arms print the same object."""
    return {"workload": WORKLOAD, "horizon": E2E_HORIZON, "parallelism": "replicas" if world > 1 else "single"}


def compact_tuned(t):
    """The autotuner's choice without its trial list."""
    if not t:
        return t
    return {k: v for k, v in t.items() if k != "trials"}


def run_reference(args, world, rank):
    """--impl reference: the reference's plugin logic on this path restated as
    multi-threaded C++ (the CPU oracle; the reference's own CUDA cannot be
    built here), on the box's host cores.  It times exactly --steps steps of
    config 1, in runs of at most 100 steps that each restart from the seeded
    state, like the GPU arm.  It loads only the oracle library: the workload's
    parameter defaults come from the oracle, never from the CUDA library."""
    if rank != 0:
        return 0
    from behavert_b200 import workloads
    from oracle import oracle
    w = workloads.large(defaults=oracle.params_default)
    threads = oracle.hardware_threads()

    def run(nsteps):
        pos, fwd, acc, feat = w.pos, w.fwd, w.acc, w.feat
        for _ in range(nsteps):
            o = oracle.step(w.params, pos, fwd, acc, feat, dt=w.dt, threads=threads, want_intermediates=False)
            pos, fwd, acc, feat = o["pos"], o["fwd"], o["acc"], o["feat"]

    run(args.warmup)
    t0 = time.perf_counter()
    for h in _horizons(args.steps):
        run(h)
    dt = time.perf_counter() - t0
    steps = args.steps
    value = w.num_agents * steps / dt
    sample = ("%d step(s) of the 1,048,576-agent config-1 workload from its seeded state (runs of at most %d "
              "steps), the GPU arm's step count" % (steps, E2E_HORIZON))
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * dt / steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded config-1 generator, numpy PCG64 seed 1)",
        "config": bench_config(world),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def cpu_baseline_leg(w, eng_state_before, gpu_state_after, budget_s=12.0):
    """Times the CPU oracle on a bounded sample and measures the GPU step's
    error against the FP64 oracle (the checker role)."""
    from oracle import oracle
    threads = oracle.hardware_threads()
    pos, fwd, acc, feat = eng_state_before
    t0 = time.perf_counter()
    steps = 0
    p, f, a, ft = pos, fwd, acc, feat
    while True:
        o = oracle.step(w.params, p, f, a, ft, dt=w.dt, threads=threads, want_intermediates=False)
        p, f, a, ft = o["pos"], o["fwd"], o["acc"], o["feat"]
        steps += 1
        if time.perf_counter() - t0 > budget_s or steps >= 20:
            break
    dt = time.perf_counter() - t0
    base = {"value": w.num_agents * steps / dt, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": "%d full step(s) of the 1,048,576-agent config-1 state (%.1f s)" % (steps, dt)}
    # error of one GPU step against FP64 and FP32 oracle steps from the same state
    o64 = oracle.step(w.params, pos.astype(np.float64), fwd.astype(np.float64), acc.astype(np.float64),
                      feat.astype(np.float64), dt=w.dt, mode=1, threads=threads, want_intermediates=False)
    gpos, gfwd, gacc, gfeat = gpu_state_after
    L = float(w.params[0].worldSize)

    def stats(x, y, periodic=False):
        """Normwise (L2) relative error, 99.99th percentile of the per-agent
        relative error, and the maximum per-agent relative error."""
        x = np.asarray(x, np.float64)
        y = np.asarray(y, np.float64)
        d = x - y
        if periodic:
            d = d - L * np.round(d / L)
        scale = np.linalg.norm(y, axis=1)
        per = np.linalg.norm(d, axis=1) / np.maximum(scale, 1e-30)
        return {"l2": float(np.linalg.norm(d) / np.linalg.norm(y)), "p9999": float(np.quantile(per, 0.9999)),
                "max": float(per.max()), "frac_over_tol": float(np.mean(per > 1e-5))}

    vel = lambda F: F[:, :3].astype(np.float64) * F[:, 3:4]
    acc_err = {"pos_vs_fp64": stats(gpos[:, :3], o64["pos"][:, :3], periodic=True),
               "vel_vs_fp64": stats(vel(gfwd), vel(o64["fwd"])),
               "feat_vs_fp64": stats(gfeat, o64["feat"]),
               "tolerance": 1e-5,
               "gate": "per quantity: normwise (l2) relative error <= tolerance and at least 99% of agents "
                       "within it on their own; p9999 and max reported (a few agents with near-cancelling steering "
                       "sums are ill-conditioned in FP32 itself; the FP32 step is bit-identical to the FP32 "
                       "oracle)"}
    qs = ("pos_vs_fp64", "vel_vs_fp64", "feat_vs_fp64")
    acc_err["within_tolerance"] = all(acc_err[k]["l2"] <= 1e-5 and acc_err[k]["frac_over_tol"] <= 1e-2 for k in qs)
    return base, acc_err


def batched_leg(device: int, steps: int = 100, loop_steps: int = 20, repeats: int = 3):
    """Config 2: 1,024 flocks of log-uniform sizes in one engine, the 100-step
    loop as one CUDA graph, against the same flocks stepped one engine per
    flock (plain per-step launches, looped over the flocks).  Both sides are
    the median of `repeats` timed runs from the seeded state."""
    import torch
    from behavert_b200 import Engine, workloads
    w = workloads.batched()
    n = w.num_agents
    dt = w.dt
    eng = Engine(w.params, device=device)
    eng.set_state(w.pos, w.fwd, w.acc)
    stream = torch.cuda.ExternalStream(eng.stream_handle())
    eng.step(dt, 3)
    tuned = eng.autotune(dt, steps=5)
    eng.step_prepare(dt, steps)
    t_batched = []
    for _ in range(repeats):
        eng.set_state(w.pos, w.fwd, w.acc)
        eng.sync()
        t_batched.append(_events_ms(stream, lambda: eng.step(dt, steps)) / 1e3)
    eng.sync()
    eng.close()
    t_batched = float(np.median(t_batched))
    # looped per-flock launches
    engines = []
    off = 0
    for p in w.params:
        e = Engine([p], device=device)
        # the full sort every step: fewer launches a step, the faster loop
        e.set_option("incremental_sort", 0)
        engines.append(e)
    t_loops = []
    for _ in range(repeats):
        off = 0
        for e, p in zip(engines, w.params):
            k = int(p.numBodies)
            e.set_state(np.ascontiguousarray(w.pos[off:off + k]), np.ascontiguousarray(w.fwd[off:off + k]),
                        np.ascontiguousarray(w.acc[off:off + k]))
            off += k
            e.step(dt, 1)
        for e in engines:
            e.sync()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(loop_steps):
            for e in engines:
                e.step(dt, 1)
        for e in engines:
            e.sync()
        t_loops.append((time.perf_counter() - t0) / loop_steps)
    for e in engines:
        e.close()
    t_loop = float(np.median(t_loops))
    batched = n * steps / t_batched
    looped = n / t_loop
    return {"workload": "config 2: %d flocks, %d agents, sizes log-uniform [128, 65536], maxNeighbors 16" %
                        (len(w.params), n),
            "value": batched, "unit": UNIT, "ms_per_step": 1e3 * t_batched / steps, "steps": steps,
            "looped_value": looped, "looped_ms_per_step": 1e3 * t_loop,
            "looped_ms_per_step_runs": [1e3 * t for t in t_loops],
            "looped": "one engine per flock (full sort each step), %d steps of plain per-step launches looped "
                      "over the flocks, median of %d runs" % (loop_steps, repeats),
            "speedup_vs_looped": batched / looped, "tuned": tuned}


def _events_ms(stream, fn):
    import torch
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    fn()
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1)


def adjoint_leg(device: int, reps: int = 5):
    """Config 3: 65,536 agents, T=50, checkpoint every 10.  Device time of
    the plain 50-step forward (one graph), the taped forward (checkpoints +
    FP64 loss) and the backward (per segment: recompute hash/sort/lists,
    reverse kernels), each the best of `reps`, on the engine's stream."""
    import torch
    from behavert_b200 import Engine, workloads
    w = workloads.adjoint()
    T, k, dt = w.steps, w.meta["checkpoint_every"], w.dt
    hidden = np.asarray([w.meta["hidden"]], np.float32)
    eng = Engine(w.params, device=device)
    stream = torch.cuda.ExternalStream(eng.stream_handle())
    eng.set_steering_weights(hidden)
    eng.set_state(w.pos, w.meta["fwd_hidden"], w.acc)
    eng.step(dt, T)
    target = eng.get_state(features=False)[0]
    eng.set_steering_weights(np.asarray([w.meta["trial"]], np.float32))
    tuned = eng.autotune(dt, steps=10)
    eng.step_prepare(dt, T)
    t_plain, t_fwd, t_bwd = [], [], []
    from behavert_b200._abi import BRT_MEM_DEVICE, check, lib, ptr
    tgt = torch.from_numpy(target).to("cuda:%d" % device)
    gw = torch.empty((1, 3), dtype=torch.float64, device=tgt.device)
    loss = torch.empty(1, dtype=torch.float64, device=tgt.device)
    h = eng.handle
    for r in range(reps + 1):
        eng.set_state(w.pos, w.fwd, w.acc)
        eng.sync()
        tp = _events_ms(stream, lambda: eng.step(dt, T))
        eng.set_state(w.pos, w.fwd, w.acc)
        eng.sync()
        tf = _events_ms(stream, lambda: check(lib().brt_adjoint_forward(h, dt, T, k, ptr(tgt), BRT_MEM_DEVICE, ptr(loss)),
                                              "adjoint_forward"))
        tb = _events_ms(stream, lambda: check(lib().brt_adjoint_backward(h, None, None, None, None, BRT_MEM_DEVICE, None,
                                                                         None, None, None, ptr(gw), BRT_MEM_DEVICE),
                                              "adjoint_backward"))
        eng.sync()
        if r:  # the first round captures the graphs
            t_plain.append(tp)
            t_fwd.append(tf)
            t_bwd.append(tb)
    eng.close()
    n = w.num_agents
    tp, tf, tb = min(t_plain), min(t_fwd), min(t_bwd)
    return {"workload": "config 3: %d agents, T=%d, checkpoint every %d, maxNeighbors 16" % (n, T, k),
            "forward_value": n * T / (tp / 1e3), "unit": UNIT,
            "adjoint_value": n * T / ((tf + tb) / 1e3),
            "ms": {"plain_forward": tp, "taped_forward": tf, "backward": tb},
            "cost_vs_forward": (tf + tb) / tp, "backward_vs_forward": tb / tp,
            "loss": float(loss.item()), "grad_weights": gw.cpu().numpy()[0].tolist(), "tuned": tuned}


def next_rows_leg(device: int, steps: int = 100, repeats: int = 3):
    """The components beside the flocking path, each on a 1,048,576-agent
    state: the Schooling law (animateSchool, and the split path with its
    random stream), the kNN neighbour semantics (useKnn: the nearest
    maxNeighbors kept), the crowd sample's order with
    steerAndSlowToAvoidNeighbors (stage-wise launches), the clustering
    analytics (10 label-propagation sweeps, then the hit rate) and a state
    snapshot.  Device time by CUDA events on the engine stream (fused steps:
    `steps`-step graphs from the seeded state, median of `repeats`).  Beside
    each, the oracle's time for the same work on the host cores, and a live
    parity check of the first step (or call) against it."""
    import os
    import tempfile
    import torch
    from behavert_b200 import Engine, workloads
    from oracle import oracle
    threads = min(oracle.hardware_threads(), 64)
    out = {}

    def fused(name, w, mode_kw):
        eng = Engine(w.params, device=device)
        stream = torch.cuda.ExternalStream(eng.stream_handle())
        eng.set_state(w.pos, w.fwd, w.acc, w.feat)
        eng.step(w.dt, 1)
        g1 = eng.get_state()
        eng.step_prepare(w.dt, steps)
        ts = []
        for _ in range(repeats + 1):
            eng.set_state(w.pos, w.fwd, w.acc, w.feat)
            eng.sync()
            ts.append(_events_ms(stream, lambda: eng.step(w.dt, steps)))
        eng.close()
        t = float(np.median(ts[1:])) / 1e3
        t0 = time.perf_counter()
        r = oracle.step(w.params, w.pos, w.fwd, w.acc, w.feat, dt=w.dt, mode=0, threads=threads,
                        want_intermediates=False, **mode_kw)
        tc = time.perf_counter() - t0
        exact = all(np.array_equal(np.asarray(a).view(np.uint32), np.ascontiguousarray(b, np.float32).view(np.uint32))
                    for a, b in ((g1[0], r["pos"]), (g1[1], r["fwd"]), (g1[2], r["acc"])))
        n = w.num_agents
        out[name] = {"value": n * steps / t, "unit": UNIT, "ms_per_step": 1e3 * t / steps,
                     "cpu_value": n / tc, "cpu_cores": threads, "cpu_sample": "1 oracle step of the same state",
                     "step1_state_bit_exact_vs_oracle": bool(exact)}

    for mode, name in ((1, "schooling_animate"), (2, "schooling_split")):
        w = workloads.schooling(n=1 << 20, L=256.0, mode=mode)
        fused(name, w, {"random_step": 1})
        out[name]["workload"] = "Schooling law (mode %d), 1,048,576 agents, cube 256, maxNeighbors 16" % mode
    w = workloads.large()
    w.params[0].useKnn = 1
    fused("knn", w, {})
    out["knn"]["workload"] = "config 1 with useKnn (the nearest 32 kept)"

    # the crowd order: stage-wise functionalities, one launch sequence a step
    w = workloads.plain(n=1 << 20, L=256.0, M=32, seed=5)
    eng = Engine(w.params, device=device)
    stream = torch.cuda.ExternalStream(eng.stream_handle())
    eng.set_state(w.pos, w.fwd, w.acc)
    eng.update_crowd(w.dt)
    g1 = eng.get_state(features=False)
    ts = []
    for _ in range(repeats + 1):
        eng.set_state(w.pos, w.fwd, w.acc)
        eng.sync()
        ts.append(_events_ms(stream, lambda: [eng.update_crowd(w.dt) for _ in range(10)]))
    t = float(np.median(ts[1:])) / 1e3 / 10
    # the clustering analytics on config 1's lists after one step
    wc = workloads.large()
    ec = Engine(wc.params, device=device)
    sc = torch.cuda.ExternalStream(ec.stream_handle())
    ec.record_lists(True)
    ec.set_state(wc.pos, wc.fwd, wc.acc, wc.feat)
    ec.step(wc.dt, 1)
    ec.computeClusterMembership(10)
    labels = ec.getClusterMembership()[:, 0].copy()
    tm, th = [], []
    for _ in range(repeats + 1):
        tm.append(_events_ms(sc, lambda: ec.computeClusterMembership(10)))
        th.append(_events_ms(sc, lambda: ec.analyzeClusterHitRate(1.5)))
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "state.brt")
        s0 = time.perf_counter()
        ec.save_snapshot(path)
        s1 = time.perf_counter()
        ec.load_snapshot(path)
        ec.sync()
        s2 = time.perf_counter()
        snap_bytes = os.path.getsize(path)
    ec.close()
    eng.close()
    t0 = time.perf_counter()
    r = oracle.step(w.params, w.pos, w.fwd, w.acc, dt=w.dt, mode=0, threads=threads, want_intermediates=False,
                    avoid_neighbors=True)
    tc = time.perf_counter() - t0
    exact = all(np.array_equal(np.asarray(a).view(np.uint32), np.ascontiguousarray(b, np.float32).view(np.uint32))
                for a, b in ((g1[0], r["pos"]), (g1[1], r["fwd"]), (g1[2], r["acc"])))
    out["crowd_avoid"] = {"workload": "crowd order (steerAndSlowToAvoidNeighbors in place of separation), "
                                      "1,048,576 agents, cube 256, maxNeighbors 32, stage-wise launches",
                          "value": w.num_agents / t, "unit": UNIT, "ms_per_step": 1e3 * t,
                          "cpu_value": w.num_agents / tc, "cpu_cores": threads,
                          "cpu_sample": "1 oracle step of the same state",
                          "step1_state_bit_exact_vs_oracle": bool(exact)}
    o = oracle.step(wc.params, wc.pos, wc.fwd, wc.acc, wc.feat, dt=wc.dt, threads=threads)
    t0 = time.perf_counter()
    ref = oracle.cluster_membership(o, 10)
    tcm = time.perf_counter() - t0
    t0 = time.perf_counter()
    oracle.cluster_hit_rate(wc.params, wc.pos, o, ref, 1.5)
    tch = time.perf_counter() - t0
    out["cluster_analytics"] = {"workload": "config 1 after one step: computeClusterMembership(10), "
                                            "analyzeClusterHitRate(1.5)",
                                "membership_ms": float(np.median(tm[1:])), "hit_rate_ms": float(np.median(th[1:])),
                                "cpu_membership_ms": 1e3 * tcm, "cpu_hit_rate_ms": 1e3 * tch,
                                "cpu_kind": "numpy restatement, 1 thread",
                                "labels_equal_vs_oracle": bool(np.array_equal(labels, ref))}
    out["snapshot"] = {"workload": "config 1 state (positions, forwards, accelerations, features)",
                       "bytes": snap_bytes, "save_ms": 1e3 * (s1 - s0), "load_ms": 1e3 * (s2 - s1),
                       "note": "host file I/O to a temporary directory"}
    return out


def adjoint_accuracy(device: int):
    """Config 3 gradients against the FP64 frozen-neighbour oracle (the CPU
    checker): the FP64 reverse with the GPU's frozen lists and branches, and
    central differences of the FP64 model at h=1e-4 (the specified step) and
    h=1e-6 (converged) on the three weights."""
    from behavert_b200 import Engine, workloads
    from oracle import oracle
    w = workloads.adjoint()
    T, k, dt = w.steps, w.meta["checkpoint_every"], float(np.float32(w.dt))
    with Engine(w.params, device=device) as eng:
        eng.set_steering_weights(np.asarray([w.meta["hidden"]], np.float32))
        eng.set_state(w.pos, w.meta["fwd_hidden"], w.acc)
        eng.step(dt, T)
        target = eng.get_state(features=False)[0]
        eng.set_steering_weights(np.asarray([w.meta["trial"]], np.float32))
        eng.set_option("adjoint_export", 1)
        eng.set_state(w.pos, w.fwd, w.acc)
        eng.adjoint_forward(target, T, k, dt)
        g = eng.adjoint_backward()
        lists, flags = eng.adjoint_tape(T)
        states = eng.adjoint_tape_states(T)
        final32 = eng.get_state(features=False)[0].astype(np.float64)
    L = float(w.params[0].worldSize)
    n = w.num_agents
    pos0, fwd0, acc0 = (a.astype(np.float64) for a in (w.pos, w.fwd, w.acc))
    w0 = np.asarray([w.meta["trial"]], np.float64)

    def loss_at(wts):
        fin = oracle.frozen_forward(w.params, pos0, fwd0, acc0, lists, weights=wts, flags=flags, dt=dt)
        d = oracle.min_image(fin["pos"][:, :3] - target[:, :3].astype(np.float64), L)
        return float(np.mean(np.sum(d * d, axis=1))), d

    _, d = loss_at(w0)
    gT = np.zeros((n, 4))
    gT[:, :3] = 2.0 * d / n
    rev = oracle.frozen_reverse(w.params, pos0, fwd0, acc0, lists, gT, weights=w0, flags=flags, dt=dt)
    f0, s0 = fwd0[:, :3], fwd0[:, 3]
    gf, gs = rev["fwd"][:, :3], rev["fwd"][:, 3]
    rev["vel"] = gs[:, None] * f0 + (gf - f0 * np.sum(f0 * gf, axis=1)[:, None]) / s0[:, None]
    out = {"grad_weights_gpu": g["weights"][0].tolist(), "grad_weights_fp64_reverse": rev["weights"][0].tolist()}
    nr = np.linalg.norm(rev["weights"][0])
    out["weights_rel_err_vs_fp64_reverse"] = float(np.linalg.norm(g["weights"][0] - rev["weights"][0]) / nr)
    # the FP64 reverse linearised at the GPU's own FP32 trajectory: the
    # adjoint's arithmetic error alone, and the trajectory's effect
    d32 = oracle.min_image(final32[:, :3] - target[:, :3].astype(np.float64), L)
    gT32 = np.zeros((n, 4))
    gT32[:, :3] = 2.0 * d32 / n
    at = oracle.frozen_reverse_at(w.params, states, lists, gT32, weights=w0, flags=flags, dt=dt)
    fa, sa = at["fwd"][:, :3], at["fwd"][:, 3]
    at["vel"] = sa[:, None] * f0 + (fa - f0 * np.sum(f0 * fa, axis=1)[:, None]) / s0[:, None]
    na = np.linalg.norm(at["weights"][0])
    out["weights_rel_err_vs_fp64_reverse_at_gpu_trajectory"] = float(np.linalg.norm(g["weights"][0] - at["weights"][0]) / na)
    out["weights_fp64_at_gpu_trajectory_vs_fp64_trajectory"] = float(np.linalg.norm(at["weights"][0] - rev["weights"][0]) / nr)
    for key in ("pos", "vel"):
        a, b = g[key][:, :3].astype(np.float64), at[key][:, :3]
        out[key + "_grad_rel_err_vs_fp64_reverse_at_gpu_trajectory"] = float(np.linalg.norm(a - b) / np.linalg.norm(b))
    for h in (1e-4, 1e-6):
        fd = np.zeros(3)
        for b in range(3):
            wp, wm = w0.copy(), w0.copy()
            wp[0, b] += h
            wm[0, b] -= h
            fd[b] = (loss_at(wp)[0] - loss_at(wm)[0]) / (2 * h)
        out["fd_h%g" % h] = fd.tolist()
        out["weights_rel_err_gpu_vs_fd_h%g" % h] = float(np.linalg.norm(g["weights"][0] - fd) / np.linalg.norm(fd))
        out["weights_rel_err_fp64_reverse_vs_fd_h%g" % h] = float(np.linalg.norm(rev["weights"][0] - fd) / np.linalg.norm(fd))
    for key in ("pos", "vel"):
        a, b = g[key][:, :3].astype(np.float64), rev[key][:, :3]
        rel = np.linalg.norm(a - b, axis=1) / np.linalg.norm(b, axis=1)
        out[key + "_grad_rel_err"] = {"median": float(np.median(rel)), "p99": float(np.quantile(rel, 0.99)),
                                      "normwise": float(np.linalg.norm(a - b) / np.linalg.norm(b))}
    return out


def fitting_leg(device: int, iters: int = 200):
    """Config 4: per-flock steering weights of 256 flocks (with 32 sphere
    obstacles each) fitted by Adam (lr 0.05) through the batched adjoint
    (libtorch autograd function), against the same iteration run one engine
    per flock."""
    import torch
    from behavert_b200 import Engine, workloads
    from behavert_b200.autograd import flock_loss
    w = workloads.fitting()
    T, k, dt = w.steps, 10, w.dt
    hidden = np.asarray(w.meta["hidden"], np.float32)
    nf = len(w.params)
    dev = torch.device("cuda:%d" % device)
    eng = Engine(w.params, device=device)
    eng.set_steering_weights(hidden)
    eng.set_state(w.pos, w.fwd, w.acc)
    eng.step(dt, T)
    tgt = torch.tensor(eng.get_state(features=False)[0][:, :3], device=dev)
    tuned = eng.autotune(dt, steps=5)
    pos0 = torch.tensor(w.pos[:, :3], device=dev)
    vel0 = torch.tensor(w.fwd[:, :3] * w.fwd[:, 3:4], device=dev)
    wt = torch.ones((nf, 3), device=dev, requires_grad=True)
    opt = torch.optim.Adam([wt], lr=w.meta["lr"])
    losses = []
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for it in range(iters):
        opt.zero_grad()
        loss = flock_loss(eng, wt, pos0, vel0, tgt, dt, T, k)
        loss.sum().backward()
        opt.step()
        if it in (0, iters - 1):
            losses.append(float(loss.detach().sum()))
    torch.cuda.synchronize()
    t_fit = time.perf_counter() - t0
    eng.close()
    err = np.abs(wt.detach().cpu().numpy() - hidden)
    rel = np.linalg.norm(wt.detach().cpu().numpy() - hidden, axis=1) / np.linalg.norm(hidden, axis=1)
    # the same iteration, one engine per flock (first iteration per engine
    # captures its graphs and is not timed)
    sizes = np.asarray(w.meta["sizes"])
    bounds = np.concatenate([[0], np.cumsum(sizes)])
    t_loop = 0.0
    for f in range(nf):
        a, b = int(bounds[f]), int(bounds[f + 1])
        e1 = Engine([w.params[f]], device=device)
        wf = torch.ones((1, 3), device=dev, requires_grad=True)
        for r in range(2):
            torch.cuda.synchronize()
            ts = time.perf_counter()
            lf = flock_loss(e1, wf, pos0[a:b], vel0[a:b], tgt[a:b], dt, T, k)
            lf.sum().backward()
            torch.cuda.synchronize()
            if r:
                t_loop += time.perf_counter() - ts
        e1.close()
    return {"workload": "config 4: %d flocks, %d agents, 32 sphere obstacles per flock (weight 2), T=%d, "
                        "checkpoint every %d, Adam lr %g" % (nf, w.num_agents, T, k, w.meta["lr"]),
            "iterations": iters, "fit_iters_per_s": iters / t_fit, "ms_per_iter": 1e3 * t_fit / iters,
            "looped_ms_per_iter": 1e3 * t_loop, "looped_fit_iters_per_s": 1.0 / t_loop,
            "speedup_vs_looped": t_loop / (t_fit / iters),
            "loss_first_last": losses,
            "recovered_weight_abs_err": {"mean": float(err.mean()), "median": float(np.median(err)),
                                         "max": float(err.max())},
            "recovered_weight_rel_err": {"median": float(np.median(rel)), "p90": float(np.quantile(rel, 0.9))},
            "tuned": tuned}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-fit", action="store_true")
    ap.add_argument("--no-next-rows", action="store_true",
                    help="skip the schooling / kNN / crowd / clustering-analytics / snapshot leg")
    ap.add_argument("--fit-iters", type=int, default=200)
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--e2e-iters", type=int, default=3)
    ap.add_argument("--profile-steps", type=int, default=0,
                    help="run W warm-up + this many single steps and exit (for ncu)")
    ap.add_argument("--profile-adjoint", type=int, default=0,
                    help="run this many config-3 adjoint iterations (taped forward + backward) and exit (for ncu)")
    ap.add_argument("--profile-fit", type=int, default=0,
                    help="run this many config-4 adjoint iterations (taped forward + backward) and exit (for ncu)")
    ap.add_argument("--profile-flocks", type=int, default=0,
                    help="with --profile-steps: step the config-2 batched workload cut to this many flocks")
    ap.add_argument("--profile-workload", default="large", choices=["large", "school1", "school2", "knn", "crowd"],
                    help="with --profile-steps: config 1 (large), the Schooling law (mode 1 or 2), config 1 with "
                         "kNN lists, or the crowd order's stage-wise step, each on 1,048,576 agents")
    ap.add_argument("--options", default="",
                    help="engine options key=value,... applied before stepping (replaces the autotuner)")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    world, rank, local = dist_setup(args)

    if args.impl == "reference":
        return run_reference(args, world, rank)

    import torch
    from behavert_b200 import Engine, workloads

    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist

    if args.profile_adjoint:
        a = workloads.adjoint()
        with Engine(a.params, device=local) as eng:
            target = np.zeros((a.num_agents, 4), np.float32)
            target[:, :3] = a.pos[:, :3]
            for _ in range(args.profile_adjoint):
                eng.set_state(a.pos, a.fwd, a.acc)
                eng.adjoint_forward(target, a.steps, a.meta["checkpoint_every"], a.dt)
                eng.adjoint_backward()
        return 0

    if args.profile_fit:
        fw = workloads.fitting()
        with Engine(fw.params, device=local) as eng:
            target = np.zeros((fw.num_agents, 4), np.float32)
            target[:, :3] = fw.pos[:, :3]
            for _ in range(args.profile_fit):
                eng.set_state(fw.pos, fw.fwd, fw.acc)
                eng.adjoint_forward(target, fw.steps, 10, fw.dt)
                eng.adjoint_backward()
        return 0

    crowd = False
    if args.profile_steps and args.profile_flocks:
        w = workloads.batched(num_flocks=args.profile_flocks)
    elif args.profile_steps and args.profile_workload in ("school1", "school2"):
        w = workloads.schooling(n=1 << 20, L=256.0, mode=int(args.profile_workload[-1]))
    elif args.profile_steps and args.profile_workload == "crowd":
        w = workloads.plain(n=1 << 20, L=256.0, M=32, seed=5)
        crowd = True
    else:
        w = workloads.large()
        if args.profile_steps and args.profile_workload == "knn":
            w.params[0].useKnn = 1
    eng = Engine(w.params, device=local)
    options = [kv.split("=") for kv in args.options.split(",") if kv]
    for key, val in options:
        eng.set_option(key, int(val))
    if options:
        args.no_autotune = True
    eng.set_state(w.pos, w.fwd, w.acc, w.feat)
    n = eng.num_agents
    dt = w.dt

    if args.profile_steps:
        for _ in range(args.warmup + args.profile_steps):
            if crowd:
                eng.update_crowd(dt)
            else:
                eng.step(dt, 1)
        eng.sync()
        eng.close()
        return 0

    stream = torch.cuda.ExternalStream(eng.stream_handle())
    from behavert_b200._abi import BRT_MEM_DEVICE, BRT_MEM_HOST, check, lib, ptr
    h = eng.handle
    dev = torch.device("cuda:%d" % local)
    # the seeded state, resident in HBM: every run of the timed region starts from it
    seeded = [torch.from_numpy(np.ascontiguousarray(x)).to(dev) for x in (w.pos, w.fwd, w.acc, w.feat)]

    def reset_to_seeded():
        check(lib().brt_set_state(h, *(ptr(x) for x in seeded), BRT_MEM_DEVICE), "set_state")

    # warm-up (single steps), the autotuner, then the graphs of the timed runs
    for _ in range(args.warmup):
        eng.step(dt, 1)
    eng.sync()
    tuned = None if args.no_autotune else eng.autotune(dt, steps=10)
    state_before = eng.get_state()
    eng.step(dt, 1)
    state_after = eng.get_state()
    horizons = _horizons(args.steps)
    for hs in sorted(set(horizons)):
        eng.step_prepare(dt, hs)
    eng.sync()

    def timed_runs():
        for hs in horizons:
            reset_to_seeded()
            check(lib().brt_step(h, dt, hs), "step")

    timed_runs()  # one untimed pass of the same sequence
    eng.sync()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    t_wall0 = time.time()
    e0.record(stream)
    timed_runs()
    e1.record(stream)
    e1.synchronize()
    t_wall1 = time.time()
    eng.sync()
    torch.cuda.synchronize()
    elapsed_ms = e0.elapsed_time(e1)
    time.sleep(0.2)
    clocks.stop()
    elapsed_ms = max_over_ranks(pg, elapsed_ms, "cuda")
    ms_per_step = elapsed_ms / args.steps
    value = replica_value(world, n, args.steps, elapsed_ms)

    # second timed pass: per-stage CUDA events (single-step launches from the seeded state)
    stage_steps = min(args.steps, E2E_HORIZON)
    reset_to_seeded()
    eng.stage_timing(True)
    for _ in range(stage_steps):
        eng.step(dt, 1)
    stage_ms, timed, launches_per_step = eng.stage_times()
    eng.stage_timing(False)
    stage_avg = [m / max(1, timed) for m in stage_ms]

    # e2e through the C-ABI with pinned host buffers: upload the seeded state,
    # run config 1's 100-step horizon, read the state back
    F = w.feat.shape[1]
    hpos, hfwd, hacc, hfeat = (torch.from_numpy(np.ascontiguousarray(x)).pin_memory()
                               for x in (w.pos, w.fwd, w.acc, w.feat))
    opos, ofwd, oacc, ofeat = (torch.empty_like(x).pin_memory() for x in (hpos, hfwd, hacc, hfeat))
    eng.step_prepare(dt, E2E_HORIZON)
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    e2 = torch.cuda.Event(enable_timing=True)
    e3 = torch.cuda.Event(enable_timing=True)
    e2.record(stream)
    for _ in range(args.e2e_iters):
        check(lib().brt_set_state(h, ptr(hpos), ptr(hfwd), ptr(hacc), ptr(hfeat), BRT_MEM_HOST), "set_state")
        check(lib().brt_step(h, dt, E2E_HORIZON), "step")
        check(lib().brt_get_state(h, ptr(opos), ptr(ofwd), ptr(oacc), ptr(ofeat), BRT_MEM_HOST), "get_state")
    e3.record(stream)
    e3.synchronize()
    e2e_ms = e2.elapsed_time(e3)
    e2e_ms = max_over_ranks(pg, e2e_ms, "cuda")
    e2e_value = replica_value(world, n, E2E_HORIZON * args.e2e_iters, e2e_ms)

    # the same timed runs with the full onesweep sort on every step (the
    # incremental re-sort off), so the radix path stays measured
    eng.set_option("incremental_sort", 0)
    for hs in sorted(set(horizons)):
        eng.step_prepare(dt, hs)
    timed_runs()
    eng.sync()
    full_sort_ms = _events_ms(stream, timed_runs) / args.steps
    eng.set_option("incremental_sort", 1)
    state_bytes = n * (16 * 3 + 4 * F)

    hbm, peak_kind = peaks()
    passes8 = math.ceil(math.log2(eng.num_cells) / 8)
    ab = alg_bytes_per_agent_step(eng.num_cells, n, F, passes8)
    fused_ms = stage_avg[3]
    fused_bytes = ab["fused_per_agent"] * n
    achieved = fused_bytes / (fused_ms / 1e3) / 1e9 if fused_ms > 0 else None
    traffic_file = ROOT / "profiles" / "flockKernel_config1_traffic.json"
    traffic = None
    warp_insts = None
    if traffic_file.exists():
        try:
            tj = json.loads(traffic_file.read_text())
            traffic = tj.get("bytes_per_launch")
            warp_insts = tj.get("warp_instructions_per_launch")
        except Exception:
            traffic = None
    # The flock kernel is bound by instruction issue, not by HBM: its ncu
    # warp-instruction count (committed beside the traffic) against the SM
    # issue peak (SMs x 4 schedulers x 1 instruction a cycle at the clock
    # sampled during the timed region), over the measured launch time.
    clock_summary = clocks.summary(t_wall0, t_wall1)
    sm_mhz = clock_summary.get("sm_mhz") or clock_summary.get("sm_max_mhz")
    sms = torch.cuda.get_device_properties(local).multi_processor_count
    issue = None
    if warp_insts and sm_mhz and fused_ms > 0:
        peak_issue = sms * 4 * sm_mhz * 1e6
        issue = {"warp_instructions_per_launch": warp_insts, "peak_warp_instructions_per_s": peak_issue,
                 "achieved_warp_instructions_per_s": warp_insts / (fused_ms / 1e3),
                 "frac": warp_insts / (fused_ms / 1e3) / peak_issue, "sm_mhz": sm_mhz, "sms": sms,
                 "source": "warp instructions from one ncu capture (profiles/flockKernel_config1_traffic.json), "
                           "time from this run's stage events"}
    step_gbs = ab["per_agent_step"] * n / (ms_per_step / 1e3) / 1e9

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded config-1 generator, numpy PCG64 seed 1)",
        "config": bench_config(world),
        "timing": {"l2": "no flush between steps: per-step working set ~%.0f MB > 126 MB L2" %
                         ((2 * state_bytes + 16 * n + 8 * eng.num_cells) / 1e6),
                   "graph": "runs of at most %d steps (config 1's horizon), each restarting from the seeded state "
                            "(a device-side state reset, inside the timed region) and launched as one CUDA graph"
                            % E2E_HORIZON},
        "tuned": compact_tuned(tuned),
        "roofline": {"bound": "hbm", "kernel": "flockKernel (fused neighbour search + steering + integration)",
                     "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": (achieved / hbm) if achieved else None, "traffic": traffic,
                     "peak_source": peak_kind,
                     "alg_bytes_per_launch": fused_bytes,
                     "step_alg_bytes_per_agent": ab["per_agent_step"],
                     "step_achieved_gbs": step_gbs, "step_frac": step_gbs / hbm,
                     "issue": issue},
        "stages_ms": {"hash": stage_avg[0], "sort": stage_avg[1], "reorder": stage_avg[2], "fused": stage_avg[3],
                      "timed_steps": timed},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": state_bytes / E2E_HORIZON,
                "d2h_bytes_per_step": state_bytes / E2E_HORIZON,
                "note": "each call: upload state, %d-step horizon, read state back" % E2E_HORIZON},
        "gpu_launches": args.steps * launches_per_step + 4 * len(horizons),
        "full_sort_ms_per_step": full_sort_ms,
        "clocks": clock_summary,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        base, accuracy = cpu_baseline_leg(w, state_before, state_after)
        line["cpu_baseline"] = base
        line["accuracy"] = accuracy
    eng.close()
    if world == 1 and not args.no_batched:
        line["batched"] = batched_leg(local)
    if world == 1 and not args.no_adjoint:
        line["adjoint"] = adjoint_leg(local)
        if rank == 0 and not args.no_cpu_baseline:
            line["adjoint"]["accuracy"] = adjoint_accuracy(local)
    if world == 1 and not args.no_fit:
        line["fitting"] = fitting_leg(local, args.fit_iters)
    if rank == 0 and world == 1 and not args.no_next_rows:
        line["next_rows"] = next_rows_leg(local)
    for leg in ("batched", "adjoint", "fitting"):
        if leg in line and isinstance(line[leg].get("tuned"), dict):
            line[leg]["tuned"] = compact_tuned(line[leg]["tuned"])
    line.update(summary_keys(line))
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)
        short = {k: v for k, v in line.items() if not isinstance(v, (dict, list))}
        sys.stderr.write("summary: %s\n" % json.dumps(short))
    return 0


def summary_keys(line: dict) -> dict:
    """Flat scalar copies of the legs' headline figures, so that a reader of
    the top level sees them without the nested objects."""
    out = {}
    iss = (line.get("roofline") or {}).get("issue")
    if iss:
        out["flock_kernel_issue_frac"] = iss["frac"]
    acc = line.get("accuracy")
    if acc:
        out["fp64_max_rel_err"] = max(acc[k]["max"] for k in ("pos_vs_fp64", "vel_vs_fp64", "feat_vs_fp64"))
        out["fp64_p9999_rel_err"] = max(acc[k]["p9999"] for k in ("pos_vs_fp64", "vel_vs_fp64", "feat_vs_fp64"))
        out["fp64_within_1e-5"] = acc["within_tolerance"]
    b = line.get("batched")
    if b:
        out["batched_agent_steps_per_s"] = b["value"]
        out["batched_ms_per_step"] = b["ms_per_step"]
        out["batched_speedup_vs_looped"] = b["speedup_vs_looped"]
    a = line.get("adjoint")
    if a:
        out["adjoint_cost_vs_forward"] = a["cost_vs_forward"]
        ac = a.get("accuracy")
        if ac:
            out["adjoint_weights_rel_err_vs_fd_h1e-06"] = ac["weights_rel_err_gpu_vs_fd_h1e-06"]
            out["adjoint_weights_rel_err_vs_fp64_reverse"] = ac["weights_rel_err_vs_fp64_reverse"]
            out["adjoint_weights_rel_err_vs_fp64_reverse_at_gpu_trajectory"] = \
                ac["weights_rel_err_vs_fp64_reverse_at_gpu_trajectory"]
            out["adjoint_trajectory_floor"] = ac["weights_fp64_at_gpu_trajectory_vs_fp64_trajectory"]
            out["adjoint_pos_grad_rel_err_normwise"] = ac["pos_grad_rel_err"]["normwise"]
            out["adjoint_vel_grad_rel_err_normwise"] = ac["vel_grad_rel_err"]["normwise"]
    f = line.get("fitting")
    if f:
        out["fit_iters_per_s"] = f["fit_iters_per_s"]
        out["fit_speedup_vs_looped"] = f["speedup_vs_looped"]
        out["fit_recovered_weight_median_abs_err"] = f["recovered_weight_abs_err"]["median"]
    nr = line.get("next_rows")
    if nr:
        for k in ("schooling_animate", "schooling_split", "knn", "crowd_avoid"):
            out[k + "_agent_steps_per_s"] = nr[k]["value"]
            out[k + "_vs_oracle_cpu"] = nr[k]["value"] / nr[k]["cpu_value"]
        out["cluster_membership_ms"] = nr["cluster_analytics"]["membership_ms"]
        out["next_rows_parity"] = all(nr[k]["step1_state_bit_exact_vs_oracle"]
                                      for k in ("schooling_animate", "schooling_split", "knn", "crowd_avoid")) \
            and nr["cluster_analytics"]["labels_equal_vs_oracle"]
    return out


if __name__ == "__main__":
    sys.exit(main())
