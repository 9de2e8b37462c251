"""Generates the oracle regression fixtures tests/golden/oracle_*.npz.

The reference ships no golden vectors for this path, so these fixtures pin the
oracle's own outputs on small seeded cases (hash/sort/cell ranges/neighbour
lists bit-exact, FP32 state bit-exact) against accidental change.  Run:
    python -m tests.golden.make_golden
"""
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def _case_plain():
    from behavert_b200 import workloads
    return workloads.plain(n=512, L=32.0, M=8, seed=21)


def _case_large():
    from behavert_b200 import workloads
    return workloads.large(n=4096, M=32, seed=22)


def _case_batched():
    from behavert_b200 import workloads
    return workloads.batched(num_flocks=5, lo=64, hi=600, seed=23, M=12)


def _case_clustering():
    from behavert_b200 import workloads
    w = workloads.plain(n=700, L=28.0, M=12, seed=24)
    rng = np.random.default_rng(24)
    p = w.params[0]
    p.featuresCount = 4
    p.clusteringForceParams[0] = 0.7
    p.alignmentClusteringForceParams[0] = 0.4
    p.featureRelaxRate = 0.05
    w.feat = rng.random((700, 4)).astype(np.float32)
    w.meta["stats"] = np.tile(np.array([0.3, 0.5, 0.7, 0.0], np.float32), (700, 1))
    return w


def _case_obstacles():
    from behavert_b200 import workloads
    w = workloads.fitting(num_flocks=2, lo=300, hi=900, seed=25, obstacles=6)
    return w


def _case_knn():
    from behavert_b200 import workloads
    w = workloads.plain(n=800, L=24.0, M=4, seed=26)
    w.params[0].useKnn = 1
    return w


CASES = {
    "oracle_plain": _case_plain,
    "oracle_large": _case_large,
    "oracle_batched": _case_batched,
    "oracle_clustering": _case_clustering,
    "oracle_obstacles": _case_obstacles,
    "oracle_knn": _case_knn,
}


def run_case(make):
    from oracle import oracle
    w = make()
    o = oracle.step(w.params, w.pos, w.fwd, w.acc, w.feat, w.meta.get("stats"), dt=0.1, mode=0, threads=1)
    out = {k: o[k] for k in ("pos", "fwd", "acc", "keys", "ids", "cell_start", "cell_end", "lists", "steer")}
    if o["feat"] is not None:
        out["feat"] = o["feat"]
    out["stats"] = o["stats"]
    return out


def main():
    for name, make in CASES.items():
        out = run_case(make)
        np.savez_compressed(HERE / (name + ".npz"), **out)
        print(name, {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main()
