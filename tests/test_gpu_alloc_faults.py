"""Allocation failures, injected on the host (gfx_fluid_debug_fail_allocation):
each device allocation of a create and of a handle's lazily allocated
workspaces fails in turn.  The call reports GFX_ERR_NO_MEMORY and leaves
nothing behind that a later call trips on: the next call allocates again,
and the handle then gives the results of a handle that never failed.  No
GPU fault is involved: the failing allocation is never made."""
import numpy as np
import pytest

from genasis_b200 import lib, problems
from genasis_b200.lib import GfxError
from tests.gpu_helpers import to_np

pytestmark = pytest.mark.gpu

NO_MEMORY = -6


def _fail(nth, variant=None):
    lib.call("gfx_fluid_debug_fail_allocation", int(nth), variant=variant)


def _raises_no_memory(fn, nth):
    _fail(nth)
    try:
        with pytest.raises(GfxError) as e:
            fn()
        assert e.value.status == NO_MEMORY, e.value
    finally:
        _fail(-1)


def test_every_allocation_of_create_can_fail():
    from genasis_b200.fluid import FluidBox

    cfg, prim = problems.sod(16)
    failed = 0
    for k in range(64):
        _fail(k)
        try:
            box = FluidBox(cfg)
        except GfxError as e:
            assert e.status == NO_MEMORY, e
            failed += 1
            continue
        finally:
            _fail(-1)
        break
    else:
        pytest.fail("create failed at every injected allocation")
    # the geometry, the nine stage buffers and the work list
    assert failed == 11
    ref = FluidBox(cfg)
    for b in (box, ref):
        b.compute_from_primitive(prim)
        for i in range(3):
            b.step(b.compute_time_step(i))
    assert np.array_equal(to_np(box.U), to_np(ref.U))
    box.close()
    ref.close()


def _pair(cfg, prim):
    from genasis_b200.fluid import FluidBox

    a, b = FluidBox(cfg), FluidBox(cfg)
    for box in (a, b):
        box.compute_from_primitive(prim)
    return a, b


def test_step_workspaces_fail_then_allocate_on_the_next_call():
    import torch

    # gravity, so that the Sources records hold the gravitational terms too
    cfg, prim = problems.rayleigh_taylor(shape=(16, 16, 32))
    a, b = _pair(cfg, prim)
    dt = b.compute_time_step(0)
    assert a.compute_time_step(0) == dt
    # Sources records: one scratch buffer
    _raises_no_memory(lambda: a.step_sources(dt), 0)
    sa, sb = a.step_sources(dt), b.step_sources(dt)
    assert np.array_equal(to_np(a.U), to_np(b.U))
    assert np.array_equal(to_np(sa), to_np(sb))
    # host step: the staging copy, the slab work list, the slab counters
    ha, hb = a.U.cpu().pin_memory(), b.U.cpu().pin_memory()
    for nth in (0, 1, 1):
        _raises_no_memory(lambda: a.step_host(ha, dt), nth)
    assert torch.equal(ha, hb)
    a.step_host(ha, dt)
    b.step_host(hb, dt)
    assert torch.equal(ha, hb)
    # tallies and the state check: one buffer each
    _raises_no_memory(lambda: a.totals(), 0)
    assert np.array_equal(a.totals(), b.totals())
    _raises_no_memory(lambda: a.check_state(), 0)
    a.check_state()
    a.close()
    b.close()


def test_adjoint_workspaces_fail_one_by_one():
    """The adjoint's workspace, its flags and its copy of the new state are
    allocated one after the other; a failure of the second or third keeps
    the ones before and the next call allocates the rest."""
    import torch

    from genasis_b200.adjoint import step_adjoint

    cfg, prim = problems.kelvin_helmholtz(16)
    a, b = _pair(cfg, prim)
    dt = b.compute_time_step(0)
    U0 = b.U.clone()
    lam1 = torch.ones_like(U0)
    for nth in (0, 1, 1):
        _raises_no_memory(lambda: step_adjoint(a, U0, dt, lam1), nth)
    la = step_adjoint(a, U0, dt, lam1)
    lb = step_adjoint(b, U0, dt, lam1)
    torch.cuda.synchronize()
    # the adjoint adds into shared cells atomically, in no fixed order
    scale = float(lb.abs().max())
    assert float((la - lb).abs().max()) <= 1e-12 * scale
    assert np.isfinite(to_np(la)).all()
    a.close()
    b.close()


def test_branch_signature_workspaces_fail_one_by_one():
    """gfx_fluid_step_branches shares the adjoint's workspace and flags and
    has a buffer of its own: each fails in turn, then the signature equals
    that of a handle that never failed."""
    from genasis_b200.adjoint import step_branches

    cfg, prim = problems.kelvin_helmholtz(16)
    a, b = _pair(cfg, prim)
    dt = b.compute_time_step(0)
    U0 = b.U.clone()
    for nth in (0, 1, 1):
        _raises_no_memory(lambda: step_branches(a, U0, dt), nth)
    ha, na, ca = step_branches(a, U0, dt)
    hb, nb, cb = step_branches(b, U0, dt)
    assert (ha, na) == (hb, nb) and np.array_equal(ca, cb)
    a.close()
    b.close()


def test_every_allocation_of_a_batch_can_fail():
    from genasis_b200.batch import FluidBatch

    bricks = problems.random_bricks(count=3, seed=5, lo=8, hi=16)
    cfgs = [c for c, _ in bricks]
    prims = [p for _, p in bricks]
    a, b = FluidBatch(cfgs), FluidBatch(cfgs)
    for x in (a, b):
        x.set_primitives(prims)
    failed = 0
    for k in range(64):
        _fail(k)
        try:
            a.evolve(n_cycles=3)
        except GfxError as e:
            assert e.status == NO_MEMORY, e
            failed += 1
            continue
        finally:
            _fail(-1)
        break
    else:
        pytest.fail("the batch failed at every injected allocation")
    assert failed == 9  # eight tables and the work list (HLL: no feature tiles)
    b.evolve(n_cycles=3)
    for ba, bb in zip(a.boxes, b.boxes):
        assert np.array_equal(to_np(ba.U), to_np(bb.U))
    a.close()
    b.close()


def test_every_allocation_of_a_chart_can_fail():
    from genasis_b200.chart import FluidChart

    cfg, prim = problems.sine_wave(16)
    failed = 0
    for k in range(256):
        _fail(k)
        try:
            a = FluidChart(cfg, (2, 2, 2))
        except GfxError as e:
            assert e.status == NO_MEMORY, e
            failed += 1
            continue
        finally:
            _fail(-1)
        break
    else:
        pytest.fail("the chart failed at every injected allocation")
    assert failed >= 80  # the allocations of its eight bricks and of its tables
    b = FluidChart(cfg, (2, 2, 2))
    for c in (a, b):
        c.from_primitive(prim)
        c.evolve(1e300, 0.0, 0, max_cycles=3)
    for ua, ub in zip(a.U, b.U):
        assert np.array_equal(to_np(ua), to_np(ub))
    a.close()
    b.close()
