"""The smallest bricks the library accepts (4 cells along an axis) and
bricks far narrower than a tile: per-step parity with the oracle and free
runs, for every boundary kind, both Riemann solvers, with gravity, through
the device step, the evolve graph and the host step."""
import numpy as np
import pytest

from genasis_b200 import problems
from genasis_b200.config import FluidConfig
from tests.gpu_helpers import assert_parity, make_pair, to_np

pytestmark = pytest.mark.gpu

BCS = [(("PERIODIC", "PERIODIC"),) * 3,
       (("REFLECTING", "OUTFLOW"), ("OUTFLOW", "REFLECTING"), ("REFLECTING", "REFLECTING")),
       (("OUTFLOW", "OUTFLOW"), ("PERIODIC", "PERIODIC"), ("REFLECTING", "OUTFLOW"))]
SHAPES = [(4, 4, 4), (4, 5, 6), (7, 4, 9), (33, 4, 5), (5, 17, 4)]


def _case(i):
    shape = SHAPES[i % len(SHAPES)]
    cfg = FluidConfig(n_cells=shape, boundary=BCS[i % len(BCS)],
                      riemann_solver="HLLC" if i % 2 == 0 else "HLL", courant_factor=0.8,
                      n_ramp_cycles=1, uniform_acceleration=0.1 if i % 3 == 2 else 0.0)
    return cfg, problems.random_state(cfg, seed=40 + i)


@pytest.mark.parametrize("i", range(len(SHAPES) * len(BCS)))
def test_small_brick_steps_match_oracle(i):
    cfg, prim = _case(i)
    box, o = make_pair(cfg, prim)
    for n in range(3):
        dt = o.timestep(n)
        o.step(dt)
        box.step(dt)
        assert_parity(to_np(box.U), o.conserved(), cfg, "small brick %d step %d" % (i, n))
    box.close()


@pytest.mark.parametrize("i", [0, 4, 7, 11])
def test_small_brick_evolve_and_host_step(i):
    """The evolve graph and the host step (on a host copy of the state) give
    the device steps' states bit for bit."""
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
    assert np.array_equal(host.numpy(), to_np(dev.U))
    assert np.array_equal(to_np(evo.U), to_np(dev.U))
    for box in (dev, evo, hst):
        box.close()
