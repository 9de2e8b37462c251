"""The CPU restatement of the BehaviorClustering analytics on hand-built
lists: label propagation is a min-label flood limited to `iterations` hops,
and the hit rate counts only close neighbours."""
import numpy as np

from behavert_b200._abi import params_default
from oracle import oracle


def _chain(n=6):
    # sorted slot s holds agent id ids[s]; slot s lists slots s-1 and s+1
    ids = np.array([3, 0, 5, 1, 4, 2], np.uint32)[:n]
    lists = np.zeros((n, 3), np.uint32)
    for s in range(n):
        nb = [t for t in (s - 1, s + 1) if 0 <= t < n]
        lists[s, 0] = len(nb)
        lists[s, 1:1 + len(nb)] = nb
    return {"ids": ids, "lists": lists}


def test_label_propagation_floods_one_hop_per_sweep():
    so = _chain()
    ids = so["ids"]
    for it in range(7):
        lab = oracle.cluster_membership(so, it)
        # the agent at sorted slot s has label max(0, s - it)
        for s in range(6):
            assert lab[ids[s]] == max(0, s - it)


def test_hit_rate_counts_close_neighbours_only():
    p = params_default()
    p.numBodies = 6
    p.worldSize = 64.0
    p.cellSize = 4.0
    so = _chain()
    ids = so["ids"]
    pos = np.zeros((6, 4), np.float32)
    # slots 0..5 along x at spacing 1, except slot 5 far away
    for s in range(6):
        pos[ids[s], :3] = (10.0 + s, 10.0, 10.0) if s < 5 else (40.0, 10.0, 10.0)
    lab = oracle.cluster_membership(so, 10)
    out = oracle.cluster_hit_rate([p], pos, so, lab, 1.5)
    # everyone reached label 0 after 10 sweeps; slot 5's only neighbour is far
    assert np.all(out[:, 0] == 0)
    assert out[ids[5], 2] == -1.0 and out[ids[5], 1] == 0.0
    for s in range(5):
        assert out[ids[s], 1] == 1.0 and out[ids[s], 2] == 0.0
