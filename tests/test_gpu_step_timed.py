"""gfx_fluid_step_timed times the kernels of an evolve cycle: after a step
of the same handle it starts from the primitives that step's stage 2 stored.
Its result equals that of gfx_fluid_step bit for bit, after an evolve, after
a step, and after the state was set from primitives.  gfx_fluid_evolve_timed
gives the evolve's results with the device time of its work."""
import numpy as np
import pytest

from genasis_b200 import problems
from tests.gpu_helpers import to_np

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("lead", ["evolve", "step", "none"])
def test_timed_step_equals_the_step(lead):
    from genasis_b200.fluid import FluidBox

    cfg, prim = problems.kelvin_helmholtz(24)
    a, b = FluidBox(cfg), FluidBox(cfg)
    for box in (a, b):
        box.compute_from_primitive(prim)
        if lead == "evolve":
            box.evolve(1.0, 0.0, 0, max_cycles=3)
        elif lead == "step":
            box.step(box.compute_time_step(0))
    dt = a.compute_time_step(3)
    for _ in range(2):
        ms = a.step_timed(dt)
        b.step(dt)
        assert len(ms) == 4 and all(m >= 0.0 for m in ms)
    assert np.array_equal(to_np(a.U), to_np(b.U))
    a.close()
    b.close()


def test_timed_evolve_equals_the_evolve():
    """gfx_fluid_evolve_timed: the same time, cycle and state as
    gfx_fluid_evolve bit for bit (from primitives, then on from an evolve),
    and device milliseconds no longer than the events around the call."""
    import torch

    from genasis_b200.fluid import FluidBox

    cfg, prim = problems.kelvin_helmholtz(24)
    a, b = FluidBox(cfg), FluidBox(cfg)
    for box in (a, b):
        box.compute_from_primitive(prim)
    t_a, c_a = a.evolve(1.0, 0.0, 0, max_cycles=4)
    t_b, c_b, ms = b.evolve_timed(1.0, 0.0, 0, max_cycles=4)
    assert (t_a, c_a) == (t_b, c_b) and ms > 0.0
    assert np.array_equal(to_np(a.U), to_np(b.U))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    t_a, c_a = a.evolve(1.0, t_a, c_a, max_cycles=9)
    t_b, c_b, ms = b.evolve_timed(1.0, t_b, c_b, max_cycles=9)
    e1.record()
    torch.cuda.synchronize()
    assert (t_a, c_a) == (t_b, c_b) and c_b == 13
    assert np.array_equal(to_np(a.U), to_np(b.U))
    assert 0.0 < ms <= e0.elapsed_time(e1)
    a.close()
    b.close()


def test_fp64_probe_rate_is_independent_of_the_chain_length():
    """The bench's FP64 probe: short and long launches give the same rate
    (within 20 %), in the range of a B200's FP64 pipes."""
    import ctypes
    import os

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    so = ctypes.CDLL(os.path.join(root, "genasis_b200", "libgfx_probe.so"))
    rates = []
    for reps, iters in ((5, 4096), (2, 4 * 4096)):
        f, ms = ctypes.c_double(), ctypes.c_double()
        assert so.gfx_probe_fp64_chains(reps, iters, ctypes.byref(f), ctypes.byref(ms)) == 0
        assert ms.value > 0.0
        rates.append(f.value)
    assert 1e12 < rates[0] < 1e14
    assert abs(rates[1] / rates[0] - 1.0) < 0.2
