"""Per-step parity with the oracle at larger bricks than the main parity file
(tens of thousands to a quarter million cells), where every stage kernel runs
many work items per SM, pencils end inside the brick and both tile shapes
take part."""
import pytest

from genasis_b200 import problems
from genasis_b200.config import FluidConfig
from tests.gpu_helpers import assert_parity, make_pair, to_np

pytestmark = pytest.mark.gpu


def _cases():
    out = []
    cfg, prim = problems.sine_wave(64, riemann_solver="HLLC")
    out.append(("sine_hllc_periodic_64", cfg, prim, 16))
    cfg, prim = problems.kelvin_helmholtz(48)
    out.append(("kh_hllc_periodic_48", cfg, prim, 8))
    cfg, prim = problems.rayleigh_taylor((32, 32, 64))
    out.append(("rt_hllc_gravity_32x32x64", cfg, prim, 8))
    cfg = FluidConfig(n_cells=(71, 45, 53), riemann_solver="HLLC",
                      boundary=(("OUTFLOW", "REFLECTING"), ("PERIODIC", "PERIODIC"),
                                ("REFLECTING", "OUTFLOW")))
    out.append(("random_hllc_mixed_71x45x53", cfg, problems.random_state(cfg, seed=31), 16))
    cfg, prim = problems.sod(64)
    out.append(("sod_hll_64", cfg, prim, 8))
    return out


CASES = _cases()
IDS = [c[0] for c in CASES]


@pytest.mark.parametrize("name,cfg,prim,rows", CASES, ids=IDS)
def test_large_brick_per_step_parity(name, cfg, prim, rows):
    box, o = make_pair(cfg, prim)
    box.set_tuning(24, 0, rows)
    for i in range(3):
        dt = o.timestep(i)
        assert box.compute_time_step(i) == pytest.approx(dt, rel=1e-14)
        o.step(dt)
        box.step(dt)
        assert_parity(to_np(box.U), o.conserved(), cfg, "%s step %d" % (name, i))
        o.set_conserved(to_np(box.U))
        o.detect_features()
    box.close()


FREE_RUNS = [
    ("kh_hllc_32", lambda: problems.kelvin_helmholtz(32), 20),
    ("rt_hllc_gravity_16x16x48", lambda: problems.rayleigh_taylor((16, 16, 48)), 20),
    ("sine_hllc_32", lambda: problems.sine_wave(32, riemann_solver="HLLC"), 20),
    ("random_hllc_shocks_30x22x26",
     lambda: (lambda c: (c, problems.random_state(c, seed=41)))(
         FluidConfig(n_cells=(30, 22, 26), riemann_solver="HLLC",
                     boundary=(("OUTFLOW", "REFLECTING"), ("PERIODIC", "PERIODIC"),
                               ("OUTFLOW", "OUTFLOW")))), 20),
]


@pytest.mark.parametrize("name,make,steps", FREE_RUNS, ids=[f[0] for f in FREE_RUNS])
def test_free_runs_stay_bitwise_in_mass_momentum_energy(name, make, steps):
    """Every operation rounds as the oracle's does (the DS field alone goes
    through log and pow, whose last bit may differ, and feeds nothing back):
    after a free run of `steps` steps with shocks, features and gravity,
    D, S1, S2, S3 and G are bit for bit the oracle's."""
    import numpy as np

    cfg, prim = make()
    box, o = make_pair(cfg, prim)
    for i in range(steps):
        dt = o.timestep(i)
        assert box.compute_time_step(i) == dt
        o.step(dt)
        box.step(dt)
    g, r = to_np(box.U), o.conserved()
    p = cfg.proper
    for f in range(5):
        assert np.array_equal(g[f][p], r[f][p]), "%s: field %d differs" % (name, f)
    box.close()
