"""The autotuner's cache file takes entries from several processes at once
(the ranks of a batch split over GPUs tune their own bricks on one host):
no entry is lost and the file stays valid JSON."""
import json
import os


def _writer(k, path):
    os.environ["GFX_TUNING_CACHE"] = path
    from genasis_b200 import autotune

    for j in range(25):
        autotune.save_entry("rank%d:key%d" % (k, j), {"z_chunk": j, "tile_rows": 8})


def test_concurrent_writers_keep_every_entry(tmp_path):
    import multiprocessing as mp

    path = str(tmp_path / "cache.json")
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_writer, args=(k, path)) for k in range(4)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    with open(path) as f:
        cache = json.load(f)
    assert len(cache) == 4 * 25
    assert cache["rank3:key24"] == {"z_chunk": 24, "tile_rows": 8}
    assert not [n for n in os.listdir(tmp_path) if n.endswith(".tmp")]


def test_cache_keys_bucket_the_workloads():
    """A brick's key rounds its edges up to multiples of 16 and names the
    solver, gravity and the fast build; a batch's key names its brick count,
    solver and a digest of every brick's size, so that a reordered or resized
    set is a different batch."""
    from genasis_b200 import autotune
    from genasis_b200.config import FluidConfig

    a = FluidConfig(n_cells=(250, 256, 241), riemann_solver="HLLC")
    assert autotune.brick_key(a) == "brick:256x256x256:HLLC:0"
    assert autotune.brick_key(a, "fast") == "brick:256x256x256:HLLC:0:fast"
    assert autotune.brick_key(a, "exact") == autotune.brick_key(a)
    g = FluidConfig(n_cells=(17, 16, 1), riemann_solver="HLL", uniform_acceleration=0.1)
    assert autotune.brick_key(g) == "brick:32x16x16:HLL:g"
    c1 = [FluidConfig(n_cells=(16, 20, 24)), FluidConfig(n_cells=(30, 16, 16))]
    c2 = list(reversed(c1))
    k1, k2 = autotune.batch_key(c1), autotune.batch_key(c2)
    assert k1.startswith("batch:2:") and k1 != k2
    assert autotune.batch_key(c1, "fast") == k1 + ":fast"
