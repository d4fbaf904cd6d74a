"""The speed build (libgfx_fluid_fast.so: fused multiply-adds, products with
rounded reciprocals, the entropy per baryon from two logarithms) against the
CPU oracle, per step from identical inputs.

Its rounding differs from the reference's, so the bar is 1e-12 relative to
the size of each conserved quantity (quantity_errors: the momentum vector's
scale for its three components); the errors under the exact build's
per-field bar are printed beside it.  The shock test recovers pressures and
velocities exactly in both builds, so the flags, which switch the flux
discontinuously, agree with the oracle's."""
import numpy as np
import pytest

from genasis_b200 import lib, problems
from genasis_b200.config import FluidConfig
from tests.gpu_helpers import PARITY_RTOL, field_errors, make_pair, quantity_errors, to_np

pytestmark = pytest.mark.gpu

FAST = "fast"


def _cases():
    out = []
    cfg, prim = problems.sod(16)
    out.append(("sod_hll_outflow_16", cfg, prim))
    cfg, prim = problems.sine_wave(32, riemann_solver="HLLC")
    out.append(("sine_hllc_periodic_32", cfg, prim))
    cfg, prim = problems.kelvin_helmholtz(32)
    out.append(("kh_hllc_periodic_32", cfg, prim))
    cfg, prim = problems.rayleigh_taylor((16, 16, 32))
    out.append(("rt_hllc_gravity_reflecting", cfg, prim))
    cfg = FluidConfig(n_cells=(37, 19, 23), riemann_solver="HLLC")
    out.append(("random_hllc_outflow_ragged", cfg, problems.random_state(cfg, seed=2)))
    cfg = FluidConfig(n_cells=(20, 33, 17), riemann_solver="HLL",
                      boundary=(("REFLECTING", "OUTFLOW"), ("OUTFLOW", "REFLECTING"),
                                ("REFLECTING", "REFLECTING")))
    out.append(("random_hll_mixed_bc", cfg, problems.random_state(cfg, seed=4)))
    cfg = FluidConfig(n_cells=(18, 12, 40), riemann_solver="HLLC",
                      boundary=(("PERIODIC", "PERIODIC"), ("OUTFLOW", "OUTFLOW"),
                                ("PERIODIC", "PERIODIC")))
    out.append(("random_hllc_mixed_periodic", cfg, problems.random_state(cfg, seed=9)))
    for k, (cfg, prim) in enumerate(problems.random_bricks(count=3, seed=20261203)):
        out.append(("random_brick_hll_%d" % k, cfg, prim))
    return out


CASES = _cases()
IDS = [c[0] for c in CASES]


@pytest.mark.parametrize("name,cfg,prim", CASES, ids=IDS)
def test_fast_build_step_parity_per_step(name, cfg, prim):
    """Four steps from identical inputs; dt and the state after each step."""
    box, o = make_pair(cfg, prim, variant=FAST)
    worst_q, worst_f = [0.0] * 6, [0.0] * 6
    for i in range(4):
        dt_o = o.timestep(i)
        dt_g = box.compute_time_step(i)
        assert dt_g == pytest.approx(dt_o, rel=1e-13), (i, dt_g, dt_o)
        o.step(dt_o)
        box.step(dt_o)
        g, r = to_np(box.U), o.conserved()
        q = quantity_errors(g, r, cfg.proper)
        assert max(q) <= PARITY_RTOL, "%s step %d: %s" % (name, i, q)
        worst_q = [max(a, b) for a, b in zip(worst_q, q)]
        worst_f = [max(a, b) for a, b in zip(worst_f, field_errors(g, r, cfg.proper))]
        o.set_conserved(g)
        o.detect_features()
        box.set_conserved(box.U.clone())
        box.detect_features()
    print(name, "fast build: per quantity", worst_q, "per field", worst_f)


@pytest.mark.parametrize("name,cfg,prim", CASES[:4], ids=IDS[:4])
def test_fast_build_shock_flags_equal_the_oracle(name, cfg, prim):
    box, o = make_pair(cfg, prim, variant=FAST)
    for i in range(2):
        dt = o.timestep(i)
        o.step(dt)
        box.step(dt)
        o.set_conserved(to_np(box.U))
        box.set_conserved(box.U.clone())
    o.detect_features()
    box.detect_features()
    f = to_np(box.features())
    ref = o.features()
    p = cfg.proper
    for d in range(3):
        assert np.array_equal(((f >> d) & 1)[p] > 0, ref[d][p] > 0), (name, d)


def test_fast_build_rejects_parabolic_reconstruction():
    from genasis_b200.fluid import FluidBox

    cfg = FluidConfig(n_cells=(8, 8, 8), reconstruction="PARABOLIC")
    with pytest.raises(lib.GfxError) as e:
        FluidBox(cfg, variant=FAST)
    assert e.value.status == -3
