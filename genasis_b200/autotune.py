"""Project-written autotuner for speed knobs that leave results unchanged
(bit for bit for the step; up to the rounding of unordered atomic additions
for the adjoint).

Knobs (gfx_fluid_set_tuning):
  tile_rows        rows of the 32-wide tile of a CTA, 8 or 16: taller tiles
                   recompute fewer y slopes and halo cells per plane, shorter
                   ones waste fewer lanes on bricks whose y extent is not a
                   multiple of 16;
  z_chunk          z length of the cell pencils a CTA of the stage kernel
                   marches: longer pencils pay fewer prologues (the two
                   planes of slopes below the pencil), shorter ones give the
                   persistent grid more items to balance;
  adjoint_segment  faces per thread in the adjoint's reverse sweep: longer
                   segments re-load fewer window cells, shorter ones give
                   more threads.

Every candidate is timed with CUDA events on a seeded state; the fastest is
kept in a JSON cache keyed by the GPU's name and a bucket of the problem
(single brick: edges rounded up to a multiple of 16, solver, gravity; batch:
the brick count and the sizes' digest).  The shipped cache, tuning/<GPU>.json,
was measured on B200s; set GFX_TUNING_CACHE to use another file.
"""
import fcntl
import hashlib
import json
import os

from . import problems
from .fluid import FluidBox, _torch

Z_CANDIDATES = (0, 8, 16, 24, 32, 48, 64, 96)
ROW_CANDIDATES = (8, 16)
SEGMENT_CANDIDATES = (4, 8, 12, 16, 32)
BATCH_Z_CANDIDATES = (8, 16, 24, 32, 48, 64, 96)
_HERE = os.path.dirname(os.path.abspath(__file__))


def gpu_name():
    torch = _torch()
    return torch.cuda.get_device_name().replace(" ", "_")


def cache_path():
    path = os.environ.get("GFX_TUNING_CACHE")
    return path if path else os.path.join(_HERE, "tuning", gpu_name() + ".json")


def load_cache():
    try:
        with open(cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def save_entry(key, entry):
    """Adds one entry to the cache file.  Ranks that tune at once on one host
    (a batch split over GPUs, each rank with its own bricks) each add their
    own key: the file is read, merged and replaced under an exclusive lock on
    a lock file beside it, through a temporary file of this process."""
    path = cache_path()
    os.makedirs(os.path.dirname(path), exist_ok=True)
    with open(path + ".lock", "a") as lock:
        fcntl.flock(lock, fcntl.LOCK_EX)
        try:
            cache = load_cache()
            cache[key] = entry
            tmp = "%s.%d.tmp" % (path, os.getpid())
            with open(tmp, "w") as f:
                json.dump(cache, f, indent=1, sort_keys=True)
            os.replace(tmp, path)
        finally:
            fcntl.flock(lock, fcntl.LOCK_UN)


def _variant_suffix(variant):
    # the exact library's entries carry no suffix; the fast build is timed
    # on its own (its kernels need fewer instructions and registers)
    return "" if (variant or "exact") == "exact" else ":" + variant


def brick_key(cfg, variant=None):
    edges = "x".join(str(16 * ((int(n) + 15) // 16)) for n in cfg.n_cells)
    grav = "g" if cfg.uniform_acceleration != 0.0 else "0"
    return "brick:%s:%s:%s%s" % (edges, cfg.riemann_solver, grav, _variant_suffix(variant))


def batch_key(cfgs, variant=None):
    sizes = ",".join("x".join(str(int(n)) for n in c.n_cells) for c in cfgs)
    digest = hashlib.sha1(sizes.encode()).hexdigest()[:12]
    return "batch:%d:%s:%s%s" % (len(cfgs), cfgs[0].riemann_solver, digest,
                                 _variant_suffix(variant))


def _time(fn, reps):
    torch = _torch()
    fn()  # warm-up (graph capture, first-touch)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    start.record()
    for _ in range(reps):
        fn()
    end.record()
    torch.cuda.synchronize()
    return start.elapsed_time(end) / reps


def tune_brick(cfg, reps=3, adjoint=True, seed=1, variant=None):
    """Times the step for every pencil length and (if adjoint) the adjoint
    step for every segment on a seeded state of cfg's size; returns
    {"z_chunk", "adjoint_segment", "ms": {...}}."""
    torch = _torch()
    from .adjoint import step_adjoint

    box = FluidBox(cfg, variant=variant)
    box.compute_from_primitive(problems.random_state(cfg, seed=seed, shocks=False))
    box.compute_from_conserved()
    U0 = box.U.clone()
    dt = box.compute_time_step(0)
    rows = ROW_CANDIDATES if cfg.reconstruction == "LINEAR" else (16,)
    ms_z = {}
    for r in rows:
        for z in Z_CANDIDATES:
            box.set_tuning(z, 0, r)

            def step():
                box.U.copy_(U0)
                box.step(dt)

            ms_z[(r, z)] = _time(step, reps)
    best_r, best_z = min(ms_z, key=ms_z.get)
    box.set_tuning(best_z, 0, best_r)
    best_seg, ms_s = 0, {}
    if adjoint and cfg.reconstruction == "LINEAR":
        box.U.copy_(U0)
        box.step(dt)
        U1 = box.U.clone()
        lam = torch.ones_like(U1)
        out = torch.empty_like(U1)
        for seg in SEGMENT_CANDIDATES:
            box.set_tuning(best_z, seg, best_r)
            ms_s[seg] = _time(lambda: step_adjoint(box, U0, dt, lam, out, U1, False), reps)
        best_seg = min(ms_s, key=ms_s.get)
    box.close()
    return {"z_chunk": best_z, "tile_rows": best_r, "adjoint_segment": best_seg,
            "ms": {"step": {"%dx%d" % k: v for k, v in ms_z.items()},
                   "adjoint": {str(k): v for k, v in ms_s.items()}}}


def tuned_box(cfg, retune=False, adjoint=True, variant=None):
    """A FluidBox of the library variant with the cached (or freshly tuned)
    knobs of cfg's bucket."""
    cache = load_cache()
    key = brick_key(cfg, variant)
    if retune or "tile_rows" not in cache.get(key, {}):
        cache[key] = tune_brick(cfg, adjoint=adjoint, variant=variant)
        save_entry(key, cache[key])
    box = FluidBox(cfg, variant=variant)
    e = cache[key]
    box.set_tuning(e["z_chunk"], e["adjoint_segment"], e["tile_rows"])
    return box


def tune_batch(batch, prims, cycles=3, retune=False):
    """Chooses the batch's tile rows and pencil length by timing whole
    batched cycles for every candidate pair (the persistent grid's balance
    depends on all bricks at once, not on one brick alone); applies and
    caches them.  The bricks' states are reset from prims afterwards.
    Returns ((tile_rows, z_chunk), ms per cycle by candidate, from_cache)."""
    cache = load_cache()
    key = batch_key([b.config for b in batch.boxes], batch.variant)
    e = cache.get(key, {})
    if not retune and "tile_rows" in e:
        batch.set_pencil_length(e["z_chunk"], e["tile_rows"])
        batch.set_primitives(prims)
        batch.set_clocks(0.0, 0)
        return (e["tile_rows"], e["z_chunk"]), e["ms"], True
    ms = {}
    batch.set_primitives(prims)
    for r in ROW_CANDIDATES:
        for z in BATCH_Z_CANDIDATES:
            # the states keep evolving from candidate to candidate: the work
            # of a cycle does not depend on them
            batch.set_pencil_length(z, r)
            ms["%dx%d" % (r, z)] = _time(lambda: batch.evolve(n_cycles=cycles), 2) / cycles
    best = min(ms, key=ms.get)
    best_r, best_z = (int(v) for v in best.split("x"))
    cache[key] = {"z_chunk": best_z, "tile_rows": best_r, "ms": ms}
    save_entry(key, cache[key])
    batch.set_pencil_length(best_z, best_r)
    batch.set_primitives(prims)
    batch.set_clocks(0.0, 0)
    return (best_r, best_z), ms, False
