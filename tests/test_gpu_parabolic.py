"""PARABOLIC reconstruction (ReconstructionType, IncrementDivergence_FV__Kernel.
f90:296-596) on the GPU against the oracle: per step from identical inputs,
free runs, the increment, bitwise mass / momentum / energy on Sod, and the
paths that keep to LINEAR reject it with GFX_ERR_UNSUPPORTED."""
import dataclasses

import numpy as np
import pytest

from genasis_b200 import problems
from genasis_b200.config import FluidConfig
from tests.gpu_helpers import assert_parity, make_pair, to_np

pytestmark = pytest.mark.gpu


def _par(cfg):
    return dataclasses.replace(cfg, reconstruction="PARABOLIC")


def _cases():
    out = []
    cfg, prim = problems.sod(16)
    out.append(("sod_hll_outflow_16", _par(cfg), prim))
    cfg, prim = problems.sine_wave(16, riemann_solver="HLLC")
    out.append(("sine_hllc_periodic_16", _par(cfg), prim))
    cfg, prim = problems.rayleigh_taylor((16, 16, 32))
    out.append(("rt_hllc_gravity_reflecting", _par(cfg), prim))
    cfg = FluidConfig(n_cells=(37, 19, 23), riemann_solver="HLLC", reconstruction="PARABOLIC")
    out.append(("random_hllc_outflow_ragged", cfg, problems.random_state(cfg, seed=2)))
    cfg = FluidConfig(n_cells=(18, 12, 40), riemann_solver="HLL", reconstruction="PARABOLIC",
                      boundary=(("PERIODIC", "PERIODIC"), ("REFLECTING", "OUTFLOW"),
                                ("PERIODIC", "PERIODIC")))
    out.append(("random_hll_mixed", cfg, problems.random_state(cfg, seed=9)))
    return out


CASES = _cases()
IDS = [c[0] for c in CASES]


@pytest.mark.parametrize("name,cfg,prim", CASES, ids=IDS)
def test_parabolic_step_parity_per_step(name, cfg, prim):
    box, o = make_pair(cfg, prim)
    for i in range(4):
        dt = o.timestep(i)
        assert box.compute_time_step(i) == pytest.approx(dt, rel=1e-14)
        o.step(dt)
        box.step(dt)
        assert_parity(to_np(box.U), o.conserved(), cfg, "%s step %d" % (name, i))
        o.set_conserved(to_np(box.U))
        o.detect_features()
    box.close()


@pytest.mark.parametrize("name,cfg,prim", CASES[:3], ids=IDS[:3])
def test_parabolic_free_run_stays_within_parity(name, cfg, prim):
    box, o = make_pair(cfg, prim)
    for i in range(6):
        dt = o.timestep(i)
        o.step(dt)
        box.step(dt)
    assert_parity(to_np(box.U), o.conserved(), cfg, name, rtol=1e-10)
    box.close()


def test_parabolic_mass_momentum_energy_bitwise_on_sod():
    cfg, prim = CASES[0][1], CASES[0][2]
    box, o = make_pair(cfg, prim)
    for i in range(3):
        dt = o.timestep(i)
        o.step(dt)
        box.step(dt)
    g, r = to_np(box.U), o.conserved()
    p = cfg.proper
    for f in range(5):
        assert np.array_equal(g[f][p], r[f][p]), "field %d differs" % f
    box.close()


@pytest.mark.parametrize("name,cfg,prim", CASES, ids=IDS)
def test_parabolic_increment_matches_oracle(name, cfg, prim):
    import torch

    box, o = make_pair(cfg, prim)
    dt = o.timestep(0)
    o.step(dt)
    box.step(dt)
    o.set_conserved(to_np(box.U))
    o.detect_features()
    box.detect_features()
    K = torch.zeros_like(box.U)
    box.increment(K, 1e-3, 0.5)
    Ko = o.increment(1e-3, 0.5)
    assert_parity(to_np(K), Ko, cfg, name)
    box.close()


def test_linear_only_paths_reject_parabolic():
    import ctypes

    import torch

    from genasis_b200 import lib
    from genasis_b200.adjoint import step_adjoint
    from genasis_b200.batch import FluidBatch
    from genasis_b200.lib import GfxError

    cfg, prim = CASES[1][1], CASES[1][2]
    box, _ = make_pair(cfg, prim)
    with pytest.raises(GfxError) as e:
        step_adjoint(box, box.U, 1e-3, torch.zeros_like(box.U))
    assert e.value.status == -3
    batch = FluidBatch([cfg])
    batch.set_primitives([prim])
    with pytest.raises(GfxError) as e:
        batch.evolve(n_cycles=1)
    assert e.value.status == -3
    c = cfg.to_c()
    rc = lib.load().gfx_fluid_step_noalloc(ctypes.byref(c), ctypes.c_void_p(box.U.data_ptr()),
                                           1e-3, 0, None, None)
    assert rc == -3
    box.close()
