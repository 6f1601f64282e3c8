"""The multi-GPU path of the benchmark is replicas (the odometry does not shard): each rank runs its own sequence
and the job's time is the slowest rank's. These tests run that host logic as two gloo ranks on the CPU."""

import os
import socket
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out):
    import datetime

    import torch.distributed as dist

    sys.path[:0] = [str(ROOT), str(ROOT / "livox-warp_b200")]
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ms = [120.0, 95.5][rank]  # the ranks' device times differ
        m = bench.max_over_ranks(ms, "cpu")
        out.put((rank, m, bench.replica_rate(580, world, m)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_replica():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    assert [g[1] for g in got] == [120.0, 120.0]
    assert all(abs(g[2] - 2 * 580 / 0.120) < 1e-6 for g in got)


def test_single_process_is_its_own_maximum():
    sys.path[:0] = [str(ROOT), str(ROOT / "livox-warp_b200")]
    import bench

    assert bench.max_over_ranks(42.0, "cpu") == 42.0
    assert bench.replica_rate(10, 1, 100.0) == pytest.approx(100.0)
