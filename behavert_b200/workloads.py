"""Seeded synthetic workloads with the shapes of the five benchmark configurations.

All randomness comes from ``numpy.random.default_rng(seed)`` (PCG64), drawn in
the order written below, so a (config, seed, size) triple always yields the
same arrays.  Positions are float32 in [0, worldSize); forward vectors are
float32 unit directions with the speed in ``w``.  ``defaults`` (plain, large)
is the function that supplies the parameter defaults: the CUDA library's
``brt_params_default`` unless a caller passes another source with the same
values (the CPU reference arm of the benchmark passes the oracle's, so that it
never loads the CUDA library).

  plain       config 0: 4,096 agents, cube 64, maxNeighbors 16, 200 steps
  large       config 1: 1,048,576 agents, cube 256, maxNeighbors 32, 70%
              uniform + 30% from 64 Gaussian blobs (sigma 6), 8 features U[0,1]
              relaxed at rate 0.05, 100 steps
  batched     config 2: 1,024 flocks, sizes log-uniform [128, 65,536], density
              1/16, per-flock weights U[0.5, 2]
  adjoint     config 3: 65,536 agents, cube 128, 50 steps
  fitting     config 4: 256 flocks, sizes log-uniform [1,024, 32,768], 32 sphere
              obstacles each, avoidance weight 2
"""
from __future__ import annotations

import dataclasses
import math
from typing import List, Optional

import numpy as np

from ._abi import BrtParams, params_default

DT = 0.1


@dataclasses.dataclass
class Workload:
    name: str
    params: List[BrtParams]
    pos: np.ndarray            # (N, 4) float32, agent-id order
    fwd: np.ndarray            # (N, 4) float32, w = speed
    acc: np.ndarray            # (N, 4) float32
    feat: Optional[np.ndarray]  # (N, F) float32 or None
    steps: int
    dt: float
    meta: dict

    @property
    def num_agents(self) -> int:
        return int(self.pos.shape[0])


def _below(x: np.ndarray, L: float) -> np.ndarray:
    """float32 values in [0, L): wrap, then push any value that rounded up to L down."""
    x = np.mod(x, L).astype(np.float32)
    top = np.nextafter(np.float32(L), np.float32(0))
    x[x >= np.float32(L)] = top
    x[x < 0] = 0
    return x


def _directions(rng, n):
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return d


def _flock_params(n, L, M, weights=(1.5, 1.0, 1.0), F=0, relax=0.0, defaults=None) -> BrtParams:
    p = (defaults or params_default)()
    p.numBodies = int(n)
    p.worldSize = float(L)
    p.cellSize = 4.0
    p.commonSearchRadius = 4.0
    p.maxNeighbors = int(M)
    p.commonMaxSpeed = 1.0
    p.commonMaxForce = 0.1
    p.commonMass = 1.0
    for arr, w in ((p.separationParams, weights[0]), (p.alignmentParams, weights[1]), (p.cohesionParams, weights[2])):
        arr[0] = float(w)
        arr[1] = 4.0
        arr[2] = -2.0
    p.featuresCount = int(F)
    p.featureRelaxRate = float(relax)
    return p


def _agents(rng, n, L):
    pos = np.zeros((n, 4), np.float32)
    pos[:, :3] = _below(rng.random((n, 3)) * L, L)
    pos[:, 3] = 1.0
    fwd = np.zeros((n, 4), np.float32)
    fwd[:, :3] = _directions(rng, n).astype(np.float32)
    fwd[:, 3] = rng.uniform(0.5, 1.0, n).astype(np.float32)
    return pos, fwd


def cube_for(n: int, density: float = 1.0 / 16.0) -> float:
    """Side of the periodic cube holding n agents at `density`, a multiple of
    the cell size 4 with at least 3 cells per side."""
    return 4.0 * max(3, int(round((n / density) ** (1.0 / 3.0) / 4.0)))


def plain(n: int = 4096, L: float = 64.0, M: int = 16, seed: int = 0, steps: int = 200, defaults=None) -> Workload:
    rng = np.random.default_rng(seed)
    pos, fwd = _agents(rng, n, L)
    acc = np.zeros((n, 4), np.float32)
    return Workload("plain", [_flock_params(n, L, M, defaults=defaults)], pos, fwd, acc, None, steps, DT,
                    {"config": 0, "seed": seed, "worldSize": L, "maxNeighbors": M})


def large(n: int = 1 << 20, L: Optional[float] = None, M: int = 32, seed: int = 1, steps: int = 100,
          blob_fraction: float = 0.3, blobs: Optional[int] = None, sigma: float = 6.0, F: int = 8,
          relax: float = 0.05, defaults=None) -> Workload:
    if L is None:
        L = 256.0 if n == (1 << 20) else 4.0 * max(3, int(round(256.0 * (n / float(1 << 20)) ** (1.0 / 3.0) / 4.0)))
    if blobs is None:
        blobs = max(1, int(round(64 * n / float(1 << 20))))
    rng = np.random.default_rng(seed)
    pos, fwd = _agents(rng, n, L)
    nb = int(round(blob_fraction * n))
    members = rng.permutation(n)[:nb]
    centres = rng.random((blobs, 3)) * L
    which = rng.integers(0, blobs, nb)
    pts = centres[which] + rng.normal(0.0, sigma, (nb, 3))
    pos[members, :3] = _below(pts, L)
    acc = np.zeros((n, 4), np.float32)
    feat = rng.random((n, F)).astype(np.float32) if F else None
    return Workload("large", [_flock_params(n, L, M, F=F, relax=relax, defaults=defaults)], pos, fwd, acc, feat,
                    steps, DT,
                    {"config": 1, "seed": seed, "worldSize": L, "maxNeighbors": M, "blobs": blobs,
                     "blob_agents": nb, "sigma": sigma, "features": F, "relax": relax})


def flock_sizes(count: int, lo: int, hi: int, rng) -> np.ndarray:
    return np.round(np.exp(rng.uniform(math.log(lo), math.log(hi), count))).astype(np.int64)


def batched(num_flocks: int = 1024, lo: int = 128, hi: int = 65536, seed: int = 2, M: int = 16,
            steps: int = 100) -> Workload:
    rng = np.random.default_rng(seed)
    sizes = flock_sizes(num_flocks, lo, hi, rng)
    weights = rng.uniform(0.5, 2.0, (num_flocks, 3))
    params, P, W = [], [], []
    for f in range(num_flocks):
        L = cube_for(int(sizes[f]))
        params.append(_flock_params(int(sizes[f]), L, M, tuple(weights[f])))
        pos, fwd = _agents(rng, int(sizes[f]), L)
        P.append(pos)
        W.append(fwd)
    pos = np.concatenate(P)
    fwd = np.concatenate(W)
    acc = np.zeros_like(pos)
    return Workload("batched", params, pos, fwd, acc, None, steps, DT,
                    {"config": 2, "seed": seed, "flocks": num_flocks, "sizes": sizes.tolist(),
                     "weights": weights.tolist(), "maxNeighbors": M})


def adjoint(n: int = 65536, L: float = 128.0, M: int = 16, seed: int = 3, steps: int = 50,
            hidden=(1.5, 1.0, 1.0), trial=(1.0, 1.0, 1.0), vel_noise: float = 0.05) -> Workload:
    rng = np.random.default_rng(seed)
    pos, fwd = _agents(rng, n, L)
    v = fwd[:, :3].astype(np.float64) * fwd[:, 3:4]
    v_trial = v + rng.normal(0.0, vel_noise, v.shape)
    sp = np.linalg.norm(v_trial, axis=1)
    fwd_trial = np.zeros_like(fwd)
    fwd_trial[:, :3] = (v_trial / sp[:, None]).astype(np.float32)
    fwd_trial[:, 3] = sp.astype(np.float32)
    acc = np.zeros((n, 4), np.float32)
    return Workload("adjoint", [_flock_params(n, L, M, trial)], pos, fwd_trial, acc, None, steps, DT,
                    {"config": 3, "seed": seed, "worldSize": L, "hidden": list(hidden), "trial": list(trial),
                     "fwd_hidden": fwd, "checkpoint_every": 10})


def fitting(num_flocks: int = 256, lo: int = 1024, hi: int = 32768, seed: int = 4, M: int = 16,
            steps: int = 40, obstacles: int = 32, avoid_weight: float = 2.0) -> Workload:
    rng = np.random.default_rng(seed)
    sizes = flock_sizes(num_flocks, lo, hi, rng)
    hidden = rng.uniform(0.5, 2.0, (num_flocks, 3))
    params, P, W = [], [], []
    for f in range(num_flocks):
        L = cube_for(int(sizes[f]))
        p = _flock_params(int(sizes[f]), L, M, (1.0, 1.0, 1.0))
        obs = np.zeros((obstacles, 4), np.float32)
        obs[:, :3] = rng.random((obstacles, 3)) * L
        obs[:, 3] = rng.uniform(2.0, 8.0, obstacles)
        p.set_obstacles(obs)
        p.obstacleAvoidanceWeight = avoid_weight
        params.append(p)
        pos, fwd = _agents(rng, int(sizes[f]), L)
        P.append(pos)
        W.append(fwd)
    pos = np.concatenate(P)
    fwd = np.concatenate(W)
    acc = np.zeros_like(pos)
    return Workload("fitting", params, pos, fwd, acc, None, steps, DT,
                    {"config": 4, "seed": seed, "flocks": num_flocks, "sizes": sizes.tolist(),
                     "hidden": hidden.tolist(), "adam_iters": 200, "lr": 0.05})


def schooling(n: int = 4096, L: float = 64.0, M: int = 16, mode: int = 1, seed: int = 5, steps: int = 50,
              random_weight: float = 0.1, flocks: int = 1) -> Workload:
    """Schooling plugin (PlugIns/Schooling) with the reference's install-time
    constants (SchoolingPlugIn.h:119-148: r_r 1, r_p = search radius, s 3,
    w_a 1, w_o 16, theta cos 0.1, eta cos 3.05); `flocks` equal flocks of n
    agents each in one engine."""
    rng = np.random.default_rng(seed)
    params, P, W = [], [], []
    for _ in range(flocks):
        p = _flock_params(n, L, M)
        p.schooling.mode = int(mode)
        p.schooling.randomDeviationWeight = float(random_weight)
        p.schooling.seed = int(rng.integers(1 << 31))
        params.append(p)
        pos, fwd = _agents(rng, n, L)
        fwd[:, 3] = p.schooling.s
        P.append(pos)
        W.append(fwd)
    pos = np.concatenate(P)
    fwd = np.concatenate(W)
    return Workload("schooling", params, pos, fwd, np.zeros_like(pos), None, steps, DT,
                    {"seed": seed, "mode": mode})


def by_name(name: str, **kw) -> Workload:
    return {"plain": plain, "large": large, "batched": batched, "adjoint": adjoint, "fitting": fitting,
            "schooling": schooling}[name](**kw)
