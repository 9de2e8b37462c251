"""Run-to-run determinism: the same seeded state stepped twice, on separate
engines, gives the same bits.  The pipeline orders its work with atomics (the
re-sort's mover lists, the adjoint's in-lists, the onesweep tile counters) and
decoupled look-back waits; the results must not depend on how those races
resolve.  Stands in for a race detector (compute-sanitizer is not available to
these tests)."""
import numpy as np
import pytest

from behavert_b200 import Engine, workloads

pytestmark = pytest.mark.gpu


def _run(w, steps, options=()):
    with Engine(w.params) as eng:
        for k, v in options:
            eng.set_option(k, v)
        eng.record_lists(True)
        eng.set_state(w.pos, w.fwd, w.acc, w.feat)
        eng.step(w.dt, steps)     # one captured graph: full sort, then incremental re-sorts
        eng.step(w.dt, 1)         # and a recorded single step
        return eng.get_state(), eng.getNeighborLists(), eng.getHash()


@pytest.mark.parametrize("name", ["large", "batched"])
def test_two_runs_give_the_same_bits(name):
    w = workloads.large() if name == "large" else workloads.batched()
    a = _run(w, 20)
    b = _run(w, 20)
    for x, y in zip(a[0], b[0]):
        if x is not None:
            assert np.array_equal(x.view(np.uint32), y.view(np.uint32))
    assert np.array_equal(a[1], b[1])
    assert np.array_equal(a[2][0], b[2][0]) and np.array_equal(a[2][1], b[2][1])


def test_full_sort_and_incremental_paths_agree_over_a_run():
    """The same 20 steps with the incremental re-sort and with the full radix
    sort on every step: the same order, lists and state."""
    w = workloads.large(n=1 << 18)
    a = _run(w, 20)
    b = _run(w, 20, [("incremental_sort", 0)])
    for x, y in zip(a[0], b[0]):
        if x is not None:
            assert np.array_equal(x.view(np.uint32), y.view(np.uint32))
    assert np.array_equal(a[1], b[1])
