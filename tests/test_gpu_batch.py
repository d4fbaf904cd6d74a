"""Batched bricks: one persistent launch per stage over many uneven bricks
gives, brick by brick, the state of the single-brick path (bit for bit) and
of the oracle (parity bar)."""
import numpy as np
import pytest

from genasis_b200 import problems
from tests.gpu_helpers import assert_parity, to_np

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("rs", ["HLL", "HLLC"])
def test_batch_matches_single_bricks_and_oracle(rs):
    from genasis_b200.batch import FluidBatch
    from genasis_b200.fluid import FluidBox
    from oracle.oracle import Oracle

    bricks = problems.random_bricks(count=7, seed=11, lo=6, hi=40, riemann_solver=rs)
    cfgs = [c for c, _ in bricks]
    prims = [p for _, p in bricks]
    batch = FluidBatch(cfgs)
    batch.set_primitives(prims)
    n_cycles = 4
    batch.evolve(n_cycles=n_cycles)
    times, cycles = batch.clocks()
    assert list(cycles) == [n_cycles] * len(bricks)
    for b, (cfg, prim) in enumerate(bricks):
        box = FluidBox(cfg)
        box.compute_from_primitive(prim)
        t, c = box.evolve(1e300, 0.0, 0, max_cycles=n_cycles)
        assert c == n_cycles and t == times[b]
        g = to_np(batch.boxes[b].U)
        assert np.array_equal(g[(slice(None),) + cfg.proper], to_np(box.U)[(slice(None),) + cfg.proper])
        o = Oracle(cfg)
        o.set_primitive(prim)
        tt = 0.0
        for i in range(n_cycles):
            dt = o.timestep(i)
            o.step(dt)
            tt += dt
        assert t == pytest.approx(tt, rel=1e-14)
        assert_parity(g, o.conserved(), cfg, "brick %d" % b, rtol=1e-10)
        box.close()
    batch.close()


def test_batch_stops_each_brick_at_its_finish_time():
    from genasis_b200.batch import FluidBatch

    bricks = problems.random_bricks(count=5, seed=3, lo=8, hi=24)
    batch = FluidBatch([c for c, _ in bricks])
    batch.set_primitives([p for _, p in bricks])
    batch.evolve(finish_time=0.01, n_cycles=1000)
    t, c = batch.clocks()
    assert np.allclose(t, 0.01, rtol=1e-14, atol=0)
    assert np.all(c >= 1)
    batch.close()


def test_batch_with_reflecting_and_periodic_faces_matches_single_bricks():
    """Bricks whose faces reverse velocities (reflecting) or wrap (periodic):
    the batched cycles, whose stage 1 copies stored primitives except where
    a boundary map reverses a velocity, equal the single-brick path bit for
    bit."""
    from genasis_b200.batch import FluidBatch
    from genasis_b200.config import FluidConfig
    from genasis_b200.fluid import FluidBox

    kinds = [(("REFLECTING", "REFLECTING"), ("PERIODIC", "PERIODIC"), ("REFLECTING", "OUTFLOW")),
             (("PERIODIC", "PERIODIC"), ("REFLECTING", "OUTFLOW"), ("PERIODIC", "PERIODIC")),
             (("OUTFLOW", "REFLECTING"), ("REFLECTING", "REFLECTING"), ("REFLECTING", "REFLECTING"))]
    shapes = [(37, 19, 23), (20, 33, 17), (45, 12, 30)]
    cfgs = [FluidConfig(n_cells=s, boundary=k, riemann_solver="HLLC", courant_factor=0.8,
                        n_ramp_cycles=1) for s, k in zip(shapes, kinds)]
    prims = [problems.random_state(c, seed=30 + i) for i, c in enumerate(cfgs)]
    batch = FluidBatch(cfgs)
    batch.set_primitives(prims)
    n_cycles = 5
    batch.evolve(n_cycles=n_cycles)
    times, cycles = batch.clocks()
    assert list(cycles) == [n_cycles] * len(cfgs)
    for b, (cfg, prim) in enumerate(zip(cfgs, prims)):
        box = FluidBox(cfg)
        box.compute_from_primitive(prim)
        t, c = box.evolve(1e300, 0.0, 0, max_cycles=n_cycles)
        assert c == n_cycles and t == times[b]
        p = (slice(None),) + cfg.proper
        assert np.array_equal(to_np(batch.boxes[b].U)[p], to_np(box.U)[p]), b
        box.close()
    batch.close()
