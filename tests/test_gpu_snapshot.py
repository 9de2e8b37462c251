"""On-disk snapshots: a run resumed from a snapshot continues bit for bit
(including the Schooling random stream), and mismatched or truncated files
are rejected."""
import numpy as np
import pytest

from behavert_b200 import workloads
from behavert_b200.engine import Engine
from behavert_b200._abi import BrtError

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["large", "schooling"])
def test_resume_is_bit_exact(tmp_path, name):
    w = workloads.large(n=1 << 14) if name == "large" else workloads.schooling(n=4096, mode=2, random_weight=0.3)
    snap = tmp_path / "state.brt"
    with Engine(w.params) as eng:
        eng.set_state(w.pos, w.fwd, w.acc, w.feat)
        eng.step(w.dt, 5)
        eng.save_snapshot(snap)
        eng.step(w.dt, 5)
        ref = eng.get_state()
    with Engine(w.params) as eng:
        eng.load_snapshot(snap)
        eng.step(w.dt, 5)
        out = eng.get_state()
    for a, b in zip(ref, out):
        if a is not None:
            assert np.array_equal(a, b)


def test_bad_snapshots_are_rejected(tmp_path):
    w = workloads.plain(n=1024, L=32.0, steps=1)
    snap = tmp_path / "state.brt"
    with Engine(w.params) as eng:
        eng.set_state(w.pos, w.fwd, w.acc)
        eng.save_snapshot(snap)
    data = snap.read_bytes()
    (tmp_path / "short.brt").write_bytes(data[: len(data) // 2])
    other = workloads.plain(n=2048, L=32.0, steps=1)
    with Engine(other.params) as eng:
        with pytest.raises(BrtError):
            eng.load_snapshot(snap)
    with Engine(w.params) as eng:
        with pytest.raises(BrtError):
            eng.load_snapshot(tmp_path / "short.brt")
        with pytest.raises(BrtError):
            eng.load_snapshot(tmp_path / "missing.brt")
