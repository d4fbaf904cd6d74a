"""The autotuner's knobs change speed only: the step and the batch give
bit-identical results for every pencil length, the adjoint the same results up
to the rounding of its unordered atomic additions; the tuner picks one of its
candidates and caches it.  Also the state check."""
import numpy as np
import pytest

from genasis_b200 import problems
from genasis_b200.config import FluidConfig
from tests.gpu_helpers import to_np

pytestmark = pytest.mark.gpu


def test_pencil_length_and_segment_leave_results_unchanged():
    import torch

    from genasis_b200.adjoint import step_adjoint
    from genasis_b200.fluid import FluidBox

    cfg = FluidConfig(n_cells=(40, 24, 37), riemann_solver="HLLC",
                      boundary=(("PERIODIC", "PERIODIC"), ("OUTFLOW", "REFLECTING"),
                                ("OUTFLOW", "OUTFLOW")))
    prim = problems.random_state(cfg, seed=4)
    ref_U = ref_lam = None
    for z, seg, rows in [(0, 0, 16), (5, 3, 8), (16, 8, 16), (37, 32, 8), (64, 1, 8)]:
        box = FluidBox(cfg)
        box.set_tuning(z, seg, rows)
        box.compute_from_primitive(prim)
        dts = []
        for i in range(3):
            dts.append(box.compute_time_step(i))
            box.step(dts[-1])
        U2 = box.U.clone()
        box.step(box.compute_time_step(3))
        lam = step_adjoint(box, U2, 1e-3, torch.ones_like(U2), None, None, True)
        torch.cuda.synchronize()
        U, L = to_np(box.U), to_np(lam)
        if ref_U is None:
            ref_U, ref_lam = U, L
        else:
            assert np.array_equal(U, ref_U), (z, seg, rows)
            # the adjoint adds into cells shared by two segments atomically, in
            # no fixed order: equal up to rounding
            scale = float(np.abs(ref_lam).max())
            assert float(np.abs(L - ref_lam).max()) <= 1e-12 * scale, (z, seg, rows)
        box.close()


def test_batch_tuner_picks_a_candidate_and_keeps_results(tmp_path, monkeypatch):
    from genasis_b200 import autotune
    from genasis_b200.batch import FluidBatch

    monkeypatch.setenv("GFX_TUNING_CACHE", str(tmp_path / "cache.json"))
    bricks = problems.random_bricks(count=6, seed=5, lo=8, hi=40)
    cfgs = [c for c, _ in bricks]
    prims = [p for _, p in bricks]
    batch = FluidBatch(cfgs)
    (rows, z), ms, cached = autotune.tune_batch(batch, prims, cycles=2)
    assert z in autotune.BATCH_Z_CANDIDATES and rows in autotune.ROW_CANDIDATES and not cached
    assert set(ms) == {"%dx%d" % (r, c) for r in autotune.ROW_CANDIDATES
                       for c in autotune.BATCH_Z_CANDIDATES}
    batch.evolve(n_cycles=3)
    tuned = [to_np(b.U) for b in batch.boxes]
    (rows2, z2), _, cached2 = autotune.tune_batch(batch, prims)
    assert cached2 and (rows2, z2) == (rows, z)
    batch.set_pencil_length(0, 16)
    batch.set_primitives(prims)
    batch.set_clocks(0.0, 0)
    batch.evolve(n_cycles=3)
    for a, b in zip(tuned, batch.boxes):
        assert np.array_equal(a, to_np(b.U))
    batch.close()


def test_check_state_reports_non_finite_values():
    import torch

    from genasis_b200.fluid import FluidBox
    from genasis_b200.lib import GfxError

    cfg, prim = problems.sod(16)
    box = FluidBox(cfg)
    box.compute_from_primitive(prim)
    box.check_state()
    bad = box.U.clone()
    g = cfg.n_ghost_layers
    bad[4, g + 3, g + 2, g + 5] = float("nan")  # a value planted on the host side
    with pytest.raises(GfxError) as e:
        box.check_state(bad)
    assert e.value.status == -4 and "1 proper cells" in str(e.value)
    torch.cuda.synchronize()
    box.close()
