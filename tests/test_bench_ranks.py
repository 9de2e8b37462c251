"""The multi-process form of bench.py (replicas, one process per GPU): the
rank reduction and the whole-job value on two gloo ranks on the CPU, and the
reference arm's rank handling (only rank 0 works and prints)."""
import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ms = 100.0 + 50.0 * rank          # rank 1 is the slow one
        dist.barrier()
        got = bench.max_over_ranks(dist, ms, "cpu")
        e2e = bench.max_over_ranks(dist, 10.0 * (world - rank), "cpu")
        value = bench.replica_value(world, 1 << 20, 100, got)
        q.put((rank, got, e2e, value))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    out = sorted(q.get(timeout=10) for _ in range(2))
    for rank, got, e2e, value in out:
        assert got == 150.0 and e2e == 20.0
        assert value == pytest.approx(2 * (1 << 20) * 100 / 0.150)


def test_single_process_keeps_its_own_time():
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.max_over_ranks(None, 12.5, "cpu") == 12.5
    assert bench.replica_value(1, 1000, 10, 1.0) == pytest.approx(1e7)


def test_reference_arm_other_ranks_exit_without_work():
    env = dict(os.environ, WORLD_SIZE="2", RANK="1", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "1", "--warmup", "3"],
                       cwd=ROOT, env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0
    assert not [l for l in r.stdout.splitlines() if l.startswith("{")]
