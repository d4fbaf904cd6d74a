"""gfx_fluid_step_timed times the kernels of an evolve cycle: after a step
of the same handle it starts from the primitives that step's stage 2 stored.
Its result equals that of gfx_fluid_step bit for bit, after an evolve, after
a step, and after the state was set from primitives."""
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
