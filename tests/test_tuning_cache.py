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
