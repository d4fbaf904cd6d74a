"""The committed fixtures of tests/golden/ (made by make_golden.py from the
oracle): the oracle must reproduce them bit for bit (CPU), and the CUDA path
must match them within the parity bar (GPU)."""
import glob
import json
import os

import numpy as np
import pytest

from genasis_b200.config import FluidConfig

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURES = sorted(glob.glob(os.path.join(HERE, "golden", "*.npz")))
IDS = [os.path.basename(f)[:-4] for f in FIXTURES]


def load(path):
    z = np.load(path)
    cfg = FluidConfig(**json.loads(str(z["config"])))
    return cfg, z


def test_fixtures_are_present():
    assert len(FIXTURES) == 4


@pytest.mark.parametrize("path", FIXTURES, ids=IDS)
def test_oracle_reproduces_the_fixture_bitwise(path):
    from oracle.oracle import Oracle

    cfg, z = load(path)
    o = Oracle(cfg)
    o.set_primitive(z["prim"])
    fl = o.new_fluence()
    for i, dt in enumerate(z["dts"]):
        assert o.timestep(i) == dt
        fl[:] = 0.0
        o.step(dt, fl)
    assert np.array_equal(o.conserved(), z["U"])
    assert np.array_equal(fl, z["fluence"])
    assert np.array_equal(o.features(), z["features"])


@pytest.mark.gpu
@pytest.mark.parametrize("path", FIXTURES, ids=IDS)
def test_cuda_path_matches_the_fixture(path):
    import torch

    from genasis_b200.fluid import FluidBox
    from tests.gpu_helpers import assert_parity, to_np

    cfg, z = load(path)
    box = FluidBox(cfg)
    box.compute_from_primitive(z["prim"])
    fl = box.new_fluence()
    for i, dt in enumerate(z["dts"]):
        assert box.compute_time_step(i) == pytest.approx(dt, rel=1e-14)
        box.step(float(dt), fl)
    torch.cuda.synchronize()
    assert_parity(to_np(box.U), z["U"], cfg, os.path.basename(path))
    f_ref = z["fluence"]
    scale = max(float(np.abs(f_ref).max()), 1e-300)
    assert float(np.abs(to_np(fl) - f_ref).max()) <= 1e-12 * scale
    flags = to_np(box.features())
    p = cfg.proper
    ref_flags = sum(((z["features"][d] > 0).astype(np.uint8) << d) for d in range(3))
    assert np.array_equal(flags[p], ref_flags[p])
    box.close()
