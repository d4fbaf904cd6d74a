"""Seeded random configurations against the oracle: brick shapes from 4 to
40 cells per axis, every boundary kind on every face, HLL and HLLC, with and
without gravity, LINEAR and PARABOLIC reconstruction, non-unit domains and
limiter parameters, states with and without jumps.  Each case takes three
steps from identical inputs with the per-step parity bar, starting with the
primitives kept at initialisation and continuing from the conserved state,
as the reference's integrator does."""
import dataclasses

import numpy as np
import pytest

from genasis_b200 import problems
from genasis_b200.config import FluidConfig
from tests.gpu_helpers import assert_parity, make_pair, to_np

pytestmark = pytest.mark.gpu

KINDS = ["OUTFLOW", "REFLECTING", "PERIODIC"]
N_CASES = 40


def _case(i):
    rng = np.random.default_rng(20261203 + i)
    shape = tuple(int(x) for x in rng.integers(4, 41, size=3))
    bounds = []
    for _ in range(3):
        k = KINDS[int(rng.integers(0, 3))]
        if k == "PERIODIC":
            bounds.append(("PERIODIC", "PERIODIC"))
        else:
            other = KINDS[int(rng.integers(0, 2))]  # OUTFLOW or REFLECTING
            bounds.append((k, other) if rng.random() < 0.5 else (other, k))
    lo = tuple(float(x) for x in rng.uniform(-1.0, 0.0, size=3))
    hi = tuple(l + float(w) for l, w in zip(lo, rng.uniform(0.5, 2.0, size=3)))
    cfg = FluidConfig(n_cells=shape, boundary=tuple(bounds), min_coordinate=lo,
                      max_coordinate=hi,
                      riemann_solver="HLLC" if rng.random() < 0.6 else "HLL",
                      reconstruction="PARABOLIC" if rng.random() < 0.2 else "LINEAR",
                      limiter_parameter=float(rng.choice([1.0, 1.4, 2.0])),
                      courant_factor=float(rng.uniform(0.3, 0.9)), n_ramp_cycles=1,
                      uniform_acceleration=float(rng.choice([0.0, 0.0, 0.1])))
    prim = problems.random_state(cfg, seed=100 + i, shocks=bool(rng.random() < 0.7))
    return cfg, prim


@pytest.mark.parametrize("i", range(N_CASES))
def test_random_configuration_matches_oracle(i):
    cfg, prim = _case(i)
    box, o = make_pair(cfg, prim)
    for n in range(3):
        dt = o.timestep(n)
        assert box.compute_time_step(n) == pytest.approx(dt, rel=1e-14)
        o.step(dt)
        box.step(dt)
        assert_parity(to_np(box.U), o.conserved(), cfg, "case %d step %d" % (i, n))
    box.close()


@pytest.mark.parametrize("i", range(0, N_CASES, 2))
def test_random_configuration_evolve_and_host_step_equal_the_steps(i):
    """The evolve graph (stored primitives, fused CFL) and the pipelined host
    step give the device steps' states bit for bit."""
    import torch

    from genasis_b200.fluid import FluidBox

    cfg, prim = _case(i)
    dev, evo, hst = FluidBox(cfg), FluidBox(cfg), FluidBox(cfg)
    for box in (dev, evo, hst):
        box.compute_from_primitive(prim)
    host = dev.U.detach().cpu().pin_memory()
    for n in range(4):
        dt = dev.compute_time_step(n)
        dev.step(dt)
        hst.step_host(host, dt)
    t, c = evo.evolve(1e300, 0.0, 0, max_cycles=4)
    torch.cuda.synchronize()
    assert c == 4
    assert np.array_equal(to_np(evo.U), to_np(dev.U))
    assert np.array_equal(host.numpy(), to_np(dev.U))
    for box in (dev, evo, hst):
        box.close()


@pytest.mark.parametrize("b", range(4))
def test_random_batches_equal_single_bricks(b):
    """Batches of random LINEAR bricks of one Riemann solver, without
    gravity and with common physical parameters (what a batch holds), evolve
    bit for bit as the single bricks."""
    import torch

    from genasis_b200.batch import FluidBatch
    from genasis_b200.fluid import FluidBox

    cases = [_case(i) for i in range(N_CASES)]
    solver = "HLLC" if b % 2 == 0 else "HLL"
    picked = [(c, p) for c, p in cases
              if c.riemann_solver == solver and c.reconstruction == "LINEAR"
              and c.uniform_acceleration == 0.0][b // 2::2][:5]
    assert len(picked) >= 3
    # a batch shares its physical parameters
    picked = [(dataclasses.replace(c, limiter_parameter=1.4, courant_factor=0.8), p)
              for c, p in picked]
    cfgs = [c for c, _ in picked]
    prims = [p for _, p in picked]
    batch = FluidBatch(cfgs)
    batch.set_primitives(prims)
    batch.evolve(n_cycles=4)
    times, cycles = batch.clocks()
    for k, (cfg, prim) in enumerate(picked):
        box = FluidBox(cfg)
        box.compute_from_primitive(prim)
        t, c = box.evolve(1e300, 0.0, 0, max_cycles=4)
        torch.cuda.synchronize()
        assert c == cycles[k] == 4 and t == times[k]
        p = (slice(None),) + cfg.proper
        assert np.array_equal(to_np(batch.boxes[k].U)[p], to_np(box.U)[p]), k
        box.close()
    batch.close()
