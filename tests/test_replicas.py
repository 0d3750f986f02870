"""The replica path of bench.py (N > 1 ranks) on CPU: two gloo ranks reduce their timings to
the slowest rank's, and the whole-job throughput counts every replica's steps."""

import datetime
import socket
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, q) -> None:
    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    import bench

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        q.put((rank, bench.reduce_max_over_ranks(10.0 + 5.0 * rank, dist, "cpu")))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_the_slowest_time():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert got == {0: 15.0, 1: 15.0}


def test_throughput_counts_every_replica():
    sys.path.insert(0, str(ROOT))
    import bench

    assert bench.reduce_max_over_ranks(3.5, None, "cpu") == 3.5
    assert bench.replica_throughput(25, 50.0, 1) == pytest.approx(500.0)
    assert bench.replica_throughput(25, 50.0, 4) == pytest.approx(2000.0)
