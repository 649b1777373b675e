"""The multi-GPU form of the benchmark is independent replicas (weak
scaling, no data-path collective): each rank solves its own copy and the job
reports all ranks' work over the slowest rank's time.  The aggregation runs
here on two gloo ranks on the CPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    import datetime
    import sys

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        bench.barrier(world)
        t_local = 0.010 * (rank + 1)          # rank 1 is the slow one
        value, t_max = bench.replica_value(1.0e6, t_local, world)
        out[rank] = (value, t_max, bench.allreduce_max(-float(rank), world))
        bench.barrier(world)
    finally:
        dist.destroy_process_group()


def test_two_replicas_report_the_slowest_rank():
    world = 2
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_rank, args=(world, _free_port(), out), nprocs=world, start_method="spawn", join=True)
    for r in range(world):
        value, t_max, m = out[r]
        assert t_max == pytest.approx(0.020)
        assert value == pytest.approx(world * 1.0e6 / 0.020)
        assert m == 0.0
