"""The batched bricks split over ranks (genasis_b200.batch.shard_bricks), run
through the bench's sharded path: two ranks, gloo on the host, both on the one
GPU of this run.  Their kernels never wait on one another (each rank advances
its own bricks; the ranks meet only in host barriers and reductions).  Every
rank's batch equals its loop of single-brick evolves bit for bit, and the
ranks report the same job figures."""
import os
import socket

import pytest

pytestmark = pytest.mark.gpu


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, cache, out):
    import datetime

    import torch
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), GFX_TUNING_CACHE=cache)
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=300))
    import bench

    line = bench.bricks_result(steps=3, warmup=3, n_bricks=12, variant="exact", world=world,
                               rank=rank)
    out[rank] = line
    dist.destroy_process_group()


def test_two_ranks_advance_disjoint_bricks_bitwise_equal_to_their_loops(tmp_path):
    import torch.multiprocessing as mp

    world = 2
    manager = mp.get_context("spawn").Manager()
    out = manager.dict()
    mp.start_processes(_rank, args=(world, _free_port(), str(tmp_path / "tuning.json"), out),
                       nprocs=world, join=True, start_method="spawn")
    a, b = out[0], out[1]
    assert a["bitwise_equal_to_plain"] is True
    assert a["n_gpus"] == 2 and a["scaling"] == "strong"
    for k in ("value", "ms_per_step", "gpu_launches", "bitwise_equal_to_plain"):
        assert a[k] == b[k], k
    assert a["config"]["bricks_this_rank"] + b["config"]["bricks_this_rank"] == 12
    assert (a["config"]["cells_this_rank"] + b["config"]["cells_this_rank"]
            == a["config"]["cells"])
    assert a["value"] > 0.0 and a["gpu_launches"] > 0
