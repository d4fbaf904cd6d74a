"""Multi-GPU runs of this path are independent replicas (one brick per rank,
no data exchange): the bench's rank logic -- barrier, max-over-ranks time and
the whole-job rate -- checked as two gloo ranks on the CPU."""
import os
import socket

import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    import bench

    bench.barrier(world)
    ms = 100.0 + 50.0 * rank  # the second replica is the slower one
    out[rank] = (bench.max_over_ranks(ms, world), bench.replica_rate(1000, 10, ms, world))
    bench.barrier(world)
    dist.destroy_process_group()


def test_two_replicas_report_the_slowest_rank_and_the_total_rate():
    import torch.multiprocessing as mp

    world = 2
    manager = mp.get_context("spawn").Manager()
    out = manager.dict()
    mp.start_processes(_rank, args=(world, _free_port(), out), nprocs=world, join=True,
                       start_method="spawn")
    for r in range(world):
        slowest, rate = out[r]
        assert slowest == 150.0
        assert rate == pytest.approx(world * 1000 * 10 / 0.150)
