"""Randomised parity sweep: seeded random configurations, each stepped twice
on the GPU and checked against the FP32 oracle fed the same state (sorted
hashes, agent order, cell ranges, neighbour lists and the FP32 state, all
bit-exact).  The draws mix what the hand-written cases cover one at a time:
1 to 3 flocks of 1 to 3,000 agents in cubes of 3 to 11 cells a side,
maxNeighbors from 1 to 40, kNN and first-M flocks side by side, a per-cell
cap, the 2D projection, features with and without relaxation, sphere
obstacles, a sensing minimum radius and angle cuts, dense clumps, coincident
agents and speeds down into the low-speed branch."""
import numpy as np
import pytest

from behavert_b200.workloads import Workload, _agents, _below, _flock_params
from tests.test_gpu_parity import check_step, make_engine

pytestmark = pytest.mark.gpu

DT = float(np.float32(0.1))


def _random_workload(seed: int) -> Workload:
    rng = np.random.default_rng(5000 + seed)
    nflocks = int(rng.choice([1, 1, 2, 3]))
    F = int(rng.choice([0, 0, 4, 8]))
    relax = float(rng.choice([0.0, 0.05]))
    params, pos, fwd, feat = [], [], [], []
    for _ in range(nflocks):
        L = 4.0 * int(rng.integers(3, 12))
        n = int(rng.integers(1, 3000))
        M = int(rng.choice([1, 4, 16, 32, 40]))
        p = _flock_params(n, L, M, weights=tuple(float(w) for w in rng.uniform(0.2, 2.0, 3)), F=F, relax=relax)
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
