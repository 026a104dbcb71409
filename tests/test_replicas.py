"""Multi-GPU is replicas only: every rank runs the whole product, the job's
step time is the maximum over ranks and its throughput the sum of the
replicas' work.  This runs bench.py's aggregation on two gloo ranks on the
CPU (no GPU)."""
import os
import sys

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank_main(rank, world, port, times, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import datetime

    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=30))
    try:
        ms = bench.replica_step_time(times[rank], "cpu")
        out[rank] = (ms, bench.replica_value(1e9, ms, world))
    finally:
        dist.destroy_process_group()


def _free_port():
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_replica_time_is_max_over_ranks_and_value_sums_replicas():
    world = 2
    times = [10.0, 15.0]
    out = mp.Manager().dict()
    mp.spawn(_rank_main, args=(world, _free_port(), times, out), nprocs=world, join=True)
    for r in range(world):
        ms, value = out[r]
        assert ms == 15.0
        assert value == pytest.approx(world * 1e9 / 0.015 / 1e9)


def test_single_process_uses_its_own_time():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.replica_step_time(12.5, "cpu") == 12.5
    assert bench.replica_value(2e9, 10.0, 1) == pytest.approx(200.0)
