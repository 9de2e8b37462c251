"""BehaviorClustering analytics on the GPU (label propagation and the cluster
hit rate) against the CPU restatement over the same step, bit-exact (labels
are integers held exactly in float32; the hit-rate distances and sums are the
same float32 operations in list order)."""
import numpy as np
import pytest

from behavert_b200 import workloads
from behavert_b200.engine import Engine
from behavert_b200._abi import BrtError

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("iterations", [0, 1, 10])
def test_membership_and_hit_rate_match_restatement(iterations):
    from oracle import oracle
    w = workloads.large(n=1 << 15, steps=1)
    with Engine(w.params) as eng:
        eng.record_lists(True)
        eng.set_state(w.pos, w.fwd, w.acc, w.feat)
        eng.step(w.dt, 1)
        eng.computeClusterMembership(iterations)
        labels = eng.getClusterMembership()
        eng.analyzeClusterHitRate(1.5)
        hr = eng.getClusterMembership()
    o = oracle.step(w.params, w.pos, w.fwd, w.acc, w.feat, dt=w.dt)
    ref_labels = oracle.cluster_membership(o, iterations)
    assert np.array_equal(labels[:, 0], ref_labels)
    ref = oracle.cluster_hit_rate(w.params, w.pos, o, ref_labels, 1.5)
    assert np.array_equal(hr[:, :3], ref[:, :3])
    if iterations == 10:
        # propagation merges labels inside the Gaussian blobs
        assert len(np.unique(labels[:, 0])) < 0.9 * w.num_agents
        assert np.all(labels[:, 0] <= ref_labels.max())


def test_membership_and_hit_rate_full_size():
    """Config 1 at full size after one step: 10 label-propagation sweeps and
    the hit rate, equal to the restatement."""
    from oracle import oracle
    w = workloads.large(steps=1)
    with Engine(w.params) as eng:
        eng.record_lists(True)
        eng.set_state(w.pos, w.fwd, w.acc, w.feat)
        eng.step(w.dt, 1)
        eng.computeClusterMembership(10)
        labels = eng.getClusterMembership()[:, 0].copy()
        eng.analyzeClusterHitRate(1.5)
        hr = eng.getClusterMembership()
    o = oracle.step(w.params, w.pos, w.fwd, w.acc, w.feat, dt=w.dt)
    ref_labels = oracle.cluster_membership(o, 10)
    assert np.array_equal(labels, ref_labels)
    ref = oracle.cluster_hit_rate(w.params, w.pos, o, ref_labels, 1.5)
    assert np.array_equal(hr[:, :3], ref[:, :3])


def test_stagewise_lists_and_errors():
    w = workloads.plain(n=2048, L=32.0, steps=1)
    with Engine(w.params) as eng:
        eng.set_state(w.pos, w.fwd, w.acc)
        with pytest.raises(BrtError):
            eng.computeClusterMembership(3)
        eng.reorderSimData()
        eng.computeNeighborhoods()
        eng.computeClusterMembership(3)
        m = eng.getClusterMembership()
    assert np.all(m[:, 0] >= 0) and np.all(m[:, 0] < w.num_agents)
