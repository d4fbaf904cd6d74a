"""Batched bricks at the sizes of the 512-brick benchmark (edges 16 to 96,
uneven, one above 64 on every axis), per step against the oracle: after each
batched cycle every brick's state agrees with the oracle's step from the
same state to the parity bar, and the brick's time step with the oracle's.
On the exact build the batch is also the single-brick path bit for bit."""
import math

import numpy as np
import pytest

from genasis_b200 import problems
from genasis_b200.config import FluidConfig
from tests.gpu_helpers import assert_parity, quantity_errors, to_np

pytestmark = pytest.mark.gpu

SIZES = [(96, 17, 80), (64, 72, 20), (16, 96, 33), (81, 40, 16), (23, 23, 96), (50, 61, 47)]


def _bricks(rs, seed=20261203):
    rng = np.random.default_rng(seed)
    out = []
    for n in SIZES:
        cfg = FluidConfig(n_cells=n, boundary=(("OUTFLOW", "OUTFLOW"),) * 3, riemann_solver=rs,
                          courant_factor=0.8, n_ramp_cycles=1)
        rho_l, p_l, rho_r, p_r = np.exp(rng.uniform(math.log(0.1), math.log(10.0), size=4))
        v_l, v_r = rng.uniform(-1.0, 1.0, size=3), rng.uniform(-1.0, 1.0, size=3)
        point = rng.uniform(0.0, 1.0, size=3)
        normal = rng.normal(size=3)
        prim = problems.riemann(cfg, rho_l, p_l, v_l, rho_r, p_r, v_r, point,
                                normal / np.linalg.norm(normal))
        out.append((cfg, prim))
    return out


@pytest.mark.parametrize("variant", ["exact", "fast"])
@pytest.mark.parametrize("rs", ["HLL", "HLLC"])
def test_batch_at_benchmark_sizes_matches_the_oracle_per_step(rs, variant):
    from genasis_b200.batch import FluidBatch
    from oracle.oracle import Oracle

    bricks = _bricks(rs)
    batch = FluidBatch([c for c, _ in bricks], variant=variant)
    batch.set_primitives([p for _, p in bricks])
    oracles = []
    for cfg, prim in bricks:
        o = Oracle(cfg)
        o.set_primitive(prim)
        oracles.append(o)
    t_prev = np.zeros(len(bricks))
    for i in range(3):
        batch.evolve(n_cycles=1)
        t, c = batch.clocks()
        assert list(c) == [i + 1] * len(bricks)
        for b, ((cfg, _), o) in enumerate(zip(bricks, oracles)):
            dt = o.timestep(i)
            assert t[b] - t_prev[b] == pytest.approx(dt, rel=1e-13), (b, i)
            o.step(t[b] - t_prev[b])
            g, r = to_np(batch.boxes[b].U), o.conserved()
            if variant == "exact":
                assert_parity(g, r, cfg, "%s brick %s step %d" % (rs, cfg.n_cells, i))
            else:
                q = quantity_errors(g, r, cfg.proper)
                assert max(q) <= 1e-12, (rs, cfg.n_cells, i, q)
            # the next step from identical inputs
            o.set_conserved(g)
            o.detect_features()
        t_prev = t.copy()
    batch.close()


def test_batch_at_benchmark_sizes_equals_single_bricks_bitwise():
    from genasis_b200.batch import FluidBatch
    from genasis_b200.fluid import FluidBox

    bricks = _bricks("HLLC", seed=5)
    batch = FluidBatch([c for c, _ in bricks])
    batch.set_primitives([p for _, p in bricks])
    batch.evolve(n_cycles=5)
    times, _ = batch.clocks()
    for b, (cfg, prim) in enumerate(bricks):
        box = FluidBox(cfg)
        box.compute_from_primitive(prim)
        t, c = box.evolve(1e300, 0.0, 0, max_cycles=5)
        assert t == times[b]
        p = (slice(None),) + cfg.proper
        assert np.array_equal(to_np(batch.boxes[b].U)[p], to_np(box.U)[p]), cfg.n_cells
        box.close()
    batch.close()
