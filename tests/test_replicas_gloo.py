"""The multi-GPU path of bench.py (independent replicas, slowest rank's time) on two
CPU ranks over gloo: no GPU involved."""
import os
import socket
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        t = bench.max_over_ranks(1.5 + rank, dist, "cpu")   # rank 1 is the slow one
        out[rank] = (t, bench.replica_rate(31, world, t))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_replicas_time_is_the_slowest_rank():
    world, port = 2, _free_port()
    out = mp.get_context("spawn").Manager().dict()
    mp.start_processes(_rank_main, args=(world, port, out), nprocs=world, start_method="spawn", join=True)
    for r in range(world):
        t, rate = out[r]
        assert t == pytest.approx(2.5)                 # max over ranks
        assert rate == pytest.approx(2 * 31 / 2.5)     # whole-job rate, weak scaling


def test_single_process_is_its_own_maximum():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(0.7, dist, "cpu") == 0.7
    assert bench.replica_rate(32, 1, 0.5) == 64.0
