"""gfx_fluid_step_host on host arrays: the pipelined path (z slabs copied in,
computed and copied back on three streams) gives the device step's result
bit for bit, state and boundary fluence, over consecutive steps, for every
kind of z boundary, with thin first slabs and with slabs of several chunks
(tall bricks).

The slabs cut z into pencils of their own.  The exact build rounds every
operation separately, so where a pencil starts does not change a bit.  The
fast build lets the compiler fuse multiply-adds, and the first face of a
pencil (computed once per work item, out of line) may fuse differently from
the faces of the plane loop; there the two paths agree to the last bits,
within 1e-14 of each quantity per run of four steps."""
import numpy as np
import pytest

from genasis_b200 import problems
from genasis_b200.config import FluidConfig
from tests.gpu_helpers import quantity_errors, to_np

pytestmark = pytest.mark.gpu


def _cases():
    kh_cfg, kh = problems.kelvin_helmholtz(16)
    kh_cfg = FluidConfig(n_cells=(20, 16, 40), boundary=(("PERIODIC", "PERIODIC"),) * 3,
                         riemann_solver="HLLC", courant_factor=0.8, n_ramp_cycles=1)
    rt_cfg, rt = problems.rayleigh_taylor(shape=(16, 12, 36), seed=2)
    mix = FluidConfig(n_cells=(18, 10, 30), riemann_solver="HLL", courant_factor=0.8,
                      n_ramp_cycles=1,
                      boundary=(("OUTFLOW", "REFLECTING"), ("PERIODIC", "PERIODIC"),
                                ("OUTFLOW", "OUTFLOW")))
    tall_p = FluidConfig(n_cells=(12, 8, 300), boundary=(("PERIODIC", "PERIODIC"),) * 3,
                         riemann_solver="HLLC", courant_factor=0.8, n_ramp_cycles=1)
    tall_o = FluidConfig(n_cells=(12, 8, 150), riemann_solver="HLLC", courant_factor=0.8,
                         n_ramp_cycles=1)
    return {
        "tall_hllc_periodic": (tall_p, problems.random_state(tall_p, seed=14)),
        "tall_hllc_outflow": (tall_o, problems.random_state(tall_o, seed=15)),
        "random_hllc_periodic": (kh_cfg, problems.random_state(kh_cfg, seed=12)),
        "rt_hllc_gravity_reflecting": (rt_cfg, rt),
        "random_hll_outflow": (mix, problems.random_state(mix, seed=13)),
    }


CASES = _cases()


@pytest.mark.parametrize("variant", ["exact", "fast"])
@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("z_chunk", [4, 16, 0])
def test_host_step_matches_the_device_step(name, z_chunk, variant):
    import torch

    from genasis_b200.fluid import FluidBox

    cfg, prim = CASES[name]
    dev, hst = FluidBox(cfg, variant=variant), FluidBox(cfg, variant=variant)
    for box in (dev, hst):
        box.set_tuning(z_chunk, 0)
        box.compute_from_primitive(prim)
    host = dev.U.detach().cpu().pin_memory()
    fl_dev = dev.new_fluence()
    fl_host = torch.zeros(tuple(fl_dev.shape), dtype=torch.float64).pin_memory()
    for i in range(4):
        dt = dev.compute_time_step(i)
        dev.step(dt, fl_dev)
        hst.step_host(host, dt, fl_host)
        torch.cuda.synchronize()
        if variant == "exact":
            assert torch.equal(host, dev.U.cpu()), (name, z_chunk, i)
            assert np.array_equal(fl_host.numpy(), to_np(fl_dev)), (name, z_chunk, i)
        else:
            every = (slice(None),) * 3
            q = quantity_errors(host.numpy(), to_np(dev.U), every)
            assert max(q) <= 1e-14, (name, z_chunk, i, q)
            f = np.abs(fl_host.numpy() - to_np(fl_dev)).max()
            assert f <= 1e-14 * max(np.abs(to_np(fl_dev)).max(), 1e-300), (name, z_chunk, i, f)
    dev.close()
    hst.close()
