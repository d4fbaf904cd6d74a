"""Multi-GPU runs of this path are independent replicas (one brick per rank,
no data exchange): the bench's rank logic -- barrier, max-over-ranks time and
the whole-job rate -- checked as two gloo ranks on the CPU.  The batched
bricks split over the ranks instead (genasis_b200.batch.shard_bricks): the
split, and the bench's reductions over it, are checked here too."""
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


def _c3_configs():
    from genasis_b200 import problems

    return [c for c, _ in problems.random_bricks(count=512, seed=20261203, only=set())]


@pytest.mark.parametrize("world", [1, 2, 3, 4, 8])
def test_the_c3_bricks_split_over_ranks_evenly(world):
    from genasis_b200.batch import shard_bricks

    cfgs = _c3_configs()
    cells = [c.n_proper for c in cfgs]
    shards = [shard_bricks(cfgs, world, r) for r in range(world)]
    every = sorted(i for sh in shards for i in sh)
    assert every == list(range(len(cfgs)))  # disjoint and complete
    loads = [sum(cells[i] for i in sh) for sh in shards]
    # greedy by decreasing size: the loads differ by at most one brick
    assert max(loads) - min(loads) <= max(cells)
    assert max(loads) <= sum(cells) / world + max(cells)
    assert shards == [shard_bricks(cfgs, world, r) for r in range(world)]  # deterministic
    with pytest.raises(ValueError):
        shard_bricks(cfgs, world, world)


def test_random_bricks_builds_only_the_selected_states_with_the_same_draws():
    import numpy as np

    from genasis_b200 import problems

    full = problems.random_bricks(count=6, seed=5, lo=8, hi=16)
    part = problems.random_bricks(count=6, seed=5, lo=8, hi=16, only={1, 4})
    for i, ((cf, pf), (cp, pp)) in enumerate(zip(full, part)):
        assert cf.n_cells == cp.n_cells
        if i in (1, 4):
            assert np.array_equal(pf, pp)
        else:
            assert pp is None


def _shard_rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    import bench
    from genasis_b200.batch import shard_bricks

    cfgs = _c3_configs()
    mine = shard_bricks(cfgs, world, rank)
    gathered = [None] * world
    dist.all_gather_object(gathered, mine)
    bench.barrier(world)
    # the bench's job figures: the slowest rank's time, every rank's launches,
    # and the batch equal to the loop only if it is on every rank
    t = bench.max_over_ranks(10.0 + rank, world)
    launches = bench.sum_over_ranks(100 + len(mine), world)
    same = bench.max_over_ranks(0.0 if rank == 0 else 1.0, world) == 0.0
    out[rank] = (gathered, t, launches, same)
    dist.destroy_process_group()


def test_two_ranks_share_the_c3_bricks_and_reduce_the_job_figures():
    import torch.multiprocessing as mp

    world = 2
    manager = mp.get_context("spawn").Manager()
    out = manager.dict()
    mp.start_processes(_shard_rank, args=(world, _free_port(), out), nprocs=world, join=True,
                       start_method="spawn")
    g0, t0, l0, s0 = out[0]
    assert out[1] == (g0, t0, l0, s0)  # every rank holds the same job figures
    assert sorted(g0[0] + g0[1]) == list(range(512)) and not set(g0[0]) & set(g0[1])
    assert t0 == 11.0
    assert l0 == 200 + 512 and isinstance(l0, int)
    assert s0 is False  # rank 1's batch differed, so the job's did
