"""Checkpoint and restart: a run interrupted by a checkpoint written to disk
and read back into a new brick ends bit for bit where the uninterrupted run
ends."""
import numpy as np
import pytest

from genasis_b200 import problems
from tests.gpu_helpers import to_np

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("maker", ["kh", "rt"])
def test_restart_continues_bitwise(tmp_path, maker):
    from genasis_b200 import checkpoint
    from genasis_b200.fluid import FluidBox

    cfg, prim = (problems.kelvin_helmholtz(16) if maker == "kh"
                 else problems.rayleigh_taylor(shape=(12, 12, 24), seed=4))
    whole = FluidBox(cfg)
    whole.compute_from_primitive(prim)
    t_w, c_w = whole.evolve(1e30, 0.0, 0, max_cycles=8)

    part = FluidBox(cfg)
    part.compute_from_primitive(prim)
    t, c = part.evolve(1e30, 0.0, 0, max_cycles=3)
    path = tmp_path / "brick.npz"
    checkpoint.save(part, path, t, c)
    part.close()
    resumed, t, c = checkpoint.load(path)
    assert c == 3
    t_r, c_r = resumed.evolve(1e30, t, c, max_cycles=5)
    assert (t_r, c_r) == (t_w, c_w)
    assert np.array_equal(to_np(resumed.U), to_np(whole.U))
    whole.close()
    resumed.close()
