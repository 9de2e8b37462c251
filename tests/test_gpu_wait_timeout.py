"""A bounded device wait that runs out is reported, and the engine stays usable.

Every decoupled look-back wait (the onesweep passes, the incremental re-sort's
cell scan) polls an unpublished predecessor at most `lookback_spin_limit`
times, then records a device error word and goes on.  The reference has no
such path: a failing CUDA call aborts the process (CUDA_SAFE_CALL,
Core/src/SimEnginePlugIn.cpp:107-112).  Here the test makes one tile's wait
run out on purpose -- option `lookback_stall_tile` has that tile poll a status
word that nothing sets, with a short limit -- and checks that the call reports
BRT_ERR_TIMEOUT, that no kernel hangs, and that the next normal step is exact.
No fault, trap or endless loop is involved: the wait gives up by design.
"""
import numpy as np
import pytest

from behavert_b200 import BrtError, Engine, workloads
from behavert_b200 import _abi
from tests.test_gpu_parity import check_step

pytestmark = pytest.mark.gpu


def _stalled_step(eng, w):
    eng.set_option("lookback_spin_limit", 2000)
    eng.set_option("lookback_stall_tile", 1)
    eng.step(w.dt, 1)
    with pytest.raises(BrtError) as ei:
        eng.sync()
    assert ei.value.status == _abi.BRT_ERR_TIMEOUT
    assert b"spin limit" in _abi.lib().brt_last_error()
    # the error word was cleared by the failing sync
    eng.sync()
    eng.set_option("lookback_stall_tile", -1)
    eng.set_option("lookback_spin_limit", 1 << 21)


@pytest.mark.parametrize("incremental", [0, 1])
def test_lookback_wait_runs_out_and_engine_recovers(incremental):
    w = workloads.large(n=65536)
    with Engine(w.params) as eng:
        eng.set_option("incremental_sort", incremental)
        eng.set_state(w.pos, w.fwd, w.acc, w.feat)
        if incremental:
            eng.step(w.dt, 1)  # the first step after set_state takes the full sort
            eng.sync()
        _stalled_step(eng, w)
        # a normal step from a known state afterwards matches the oracle exactly
        eng.set_state(w.pos, w.fwd, w.acc, w.feat)
        check_step(eng, w.params)
        check_step(eng, w.params)  # (with incremental 1: the re-sort path)


def test_graph_with_stalled_wait_reports_timeout():
    """The same inside a captured multi-step graph: the error surfaces at the
    next sync, and the graph cache is rebuilt when the options change."""
    w = workloads.large(n=65536)
    with Engine(w.params) as eng:
        eng.set_state(w.pos, w.fwd, w.acc, w.feat)
        eng.set_option("lookback_spin_limit", 500)
        eng.set_option("lookback_stall_tile", 2)
        eng.step(w.dt, 5)
        with pytest.raises(BrtError) as ei:
            eng.sync()
        assert ei.value.status == _abi.BRT_ERR_TIMEOUT
        eng.set_option("lookback_stall_tile", -1)
        eng.set_option("lookback_spin_limit", 1 << 21)
        eng.set_state(w.pos, w.fwd, w.acc, w.feat)
        eng.step(w.dt, 5)
        eng.sync()
        check_step(eng, w.params)


def test_wait_options_are_validated():
    w = workloads.plain(n=1000, L=40.0)
    with Engine(w.params) as eng:
        for key, val in (("lookback_spin_limit", -1), ("lookback_stall_tile", -2)):
            with pytest.raises(BrtError) as ei:
                eng.set_option(key, val)
            assert ei.value.status == _abi.BRT_ERR_ARG
