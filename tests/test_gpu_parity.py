"""Parity of the CUDA path (called through the C ABI) with the CPU oracle on
the same seeded inputs, per step, at sizes the oracle finishes in seconds."""
import numpy as np
import pytest

from genasis_b200 import problems
from genasis_b200.config import FluidConfig
from oracle.oracle import Oracle
from tests.gpu_helpers import PARITY_RTOL, assert_parity, field_errors, make_pair, to_np

pytestmark = pytest.mark.gpu


def _cases():
    """(name, config, primitive initial state) of the parity cases."""
    out = []
    cfg, prim = problems.sod(16)
    out.append(("sod_hll_outflow_16", cfg, prim))
    cfg, prim = problems.sine_wave(16, riemann_solver="HLLC")
    out.append(("sine_hllc_periodic_16", cfg, prim))
    cfg, prim = problems.kelvin_helmholtz(16)
    out.append(("kh_hllc_periodic_16", cfg, prim))
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
    cfg, prim = problems.random_bricks(count=3, seed=20261203)[2]
    out.append(("random_brick_hll", cfg, prim))
    return out


CASES = _cases()
IDS = [c[0] for c in CASES]


@pytest.mark.parametrize("name,cfg,prim", CASES, ids=IDS)
def test_from_primitive_matches_oracle(name, cfg, prim):
    box, o = make_pair(cfg, prim)
    every = (slice(None),) * 3
    assert_parity(to_np(box.U), o.conserved(), cfg, name, rtol=1e-15, index=every)


@pytest.mark.parametrize("name,cfg,prim", CASES, ids=IDS)
def test_step_parity_per_step(name, cfg, prim):
    """Five RK2 steps from identical inputs: the state and the CFL time step
    after every step agree with the oracle to the parity bar."""
    box, o = make_pair(cfg, prim)
    worst = [0.0] * 6
    for i in range(5):
        dt_o = o.timestep(i)
        dt_g = box.compute_time_step(i)
        assert dt_g == pytest.approx(dt_o, rel=1e-14), (i, dt_g, dt_o)
        o.step(dt_o)
        box.step(dt_o)
        errs = assert_parity(to_np(box.U), o.conserved(), cfg, "%s step %d" % (name, i))
        worst = [max(a, b) for a, b in zip(worst, errs)]
        # resynchronise so each step starts from identical inputs
        o.set_conserved(to_np(box.U))
        o.detect_features()
    print(name, "worst relative error per field", worst)


@pytest.mark.parametrize("name,cfg,prim", CASES[:5], ids=IDS[:5])
def test_free_run_stays_within_parity(name, cfg, prim):
    box, o = make_pair(cfg, prim)
    for i in range(8):
        dt = o.timestep(i)
        o.step(dt)
        box.step(dt)
    assert_parity(to_np(box.U), o.conserved(), cfg, name, rtol=1e-10)


def test_mass_momentum_energy_bitwise_on_sod():
    """Both sides round every operation identically: D, S and G match bit for
    bit (DS goes through log / pow, whose last bit may differ)."""
    cfg, prim = problems.sod(16)
    box, o = make_pair(cfg, prim)
    for i in range(3):
        dt = o.timestep(i)
        o.step(dt)
        box.step(dt)
    g, r = to_np(box.U), o.conserved()
    p = cfg.proper
    for f in range(5):
        assert np.array_equal(g[f][p], r[f][p]), "field %d differs" % f


@pytest.mark.parametrize("name,cfg,prim", CASES, ids=IDS)
def test_ghosts_match_oracle_after_step(name, cfg, prim):
    box, o = make_pair(cfg, prim)
    for i in range(2):
        dt = o.timestep(i)
        o.step(dt)
        box.step(dt)
    every = (slice(None),) * 3
    assert_parity(to_np(box.U), o.conserved(), cfg, name, rtol=1e-12, index=every)


@pytest.mark.parametrize("name,cfg,prim", CASES, ids=IDS)
def test_increment_matches_oracle(name, cfg, prim):
    """IncrementDivergence_FV % Compute: all six fields and the fluence."""
    import torch

    box, o = make_pair(cfg, prim)
    # a state with features: take one step first, then detect on both sides
    dt = o.timestep(0)
    o.step(dt)
    box.step(dt)
    o.set_conserved(to_np(box.U))
    o.detect_features()
    box.detect_features()
    K = torch.zeros_like(box.U)
    fl = box.new_fluence()
    box.increment(K, 1.3e-3, 0.5, fl)
    fl_o = o.new_fluence()
    Ko = o.increment(1.3e-3, 0.5, fluence=fl_o)
    assert_parity(to_np(K), Ko, cfg, name + " K")
    errs = [float(np.abs(to_np(fl)[f] - fl_o[f]).max() / max(np.abs(fl_o[f]).max(), 1e-300))
            for f in range(6)]
    assert max(errs) <= PARITY_RTOL, errs


@pytest.mark.parametrize("name,cfg,prim", CASES[:5], ids=IDS[:5])
def test_features_match_oracle(name, cfg, prim):
    box, o = make_pair(cfg, prim)
    for i in range(2):
        dt = o.timestep(i)
        o.step(dt)
        box.step(dt)
    f = to_np(box.features())
    ref = o.features()
    p = cfg.proper
    for d in range(3):
        assert np.array_equal(((f >> d) & 1)[p] > 0, ref[d][p] > 0), d


def test_step_fluence_matches_oracle():
    cfg = FluidConfig(n_cells=(21, 14, 11), riemann_solver="HLLC")
    box, o = make_pair(cfg, problems.random_state(cfg, seed=12))
    fl = box.new_fluence()
    fl_o = o.new_fluence()
    dt = o.timestep(4)
    o.step(dt, fl_o)
    box.step(dt, fl)
    g = to_np(fl)
    errs = [float(np.abs(g[f] - fl_o[f]).max() / max(np.abs(fl_o[f]).max(), 1e-300))
            for f in range(6)]
    assert max(errs) <= PARITY_RTOL, errs


def test_to_primitive_matches_oracle():
    cfg = FluidConfig(n_cells=(13, 9, 10), riemann_solver="HLLC")
    box, o = make_pair(cfg, problems.random_state(cfg, seed=21))
    U = to_np(box.U).copy()
    U[4][cfg.proper][0, 0, :3] = -1.0  # negative internal energy -> floor
    U[0][cfg.proper][1, 1, :2] = -0.5  # negative density -> zero state
    import torch

    box.U.copy_(torch.as_tensor(U))
    o.set_conserved(U)
    prim, aux = box.compute_from_conserved(primitive=True, aux=True)
    every = (slice(None),) * 3
    assert_parity(to_np(box.U), o.conserved(), cfg, "floored U", index=every)
    assert_parity(to_np(prim), o.primitive(), cfg, "primitive", index=every)
    ref_aux = o.aux()
    assert np.array_equal(to_np(aux)[0], ref_aux[0])  # pressure
    assert np.array_equal(to_np(aux)[1], ref_aux[1])  # sound speed


def test_evolve_matches_oracle_loop():
    cfg, prim = problems.sine_wave(16, riemann_solver="HLLC")
    box, o = make_pair(cfg, prim)
    finish = 0.03
    t, c = box.evolve(finish, 0.0, 0)
    tt, i = 0.0, 0
    while tt < finish:
        dt = o.timestep(i)
        if tt + dt > finish:
            dt = finish - tt
        o.step(dt)
        tt += dt
        i += 1
    assert c == i
    assert t == pytest.approx(tt, rel=1e-15)
    assert_parity(to_np(box.U), o.conserved(), cfg, "evolve", rtol=1e-10)


def test_step_host_matches_device_step():
    import torch

    cfg, prim = problems.kelvin_helmholtz(16)
    box, _ = make_pair(cfg, prim)
    box2, _ = make_pair(cfg, prim)
    host = box.U.detach().cpu().pin_memory()
    dt = box.compute_time_step(0)
    box.step(dt)
    box2.step_host(host, dt)
    torch.cuda.synchronize()
    assert torch.equal(host, box.U.cpu())


def test_errors_are_reported_not_raised_on_device():
    from genasis_b200 import GfxError
    from genasis_b200.fluid import FluidBox

    with pytest.raises(GfxError):
        FluidBox(FluidConfig(n_cells=(2, 8, 8)))
    with pytest.raises(GfxError):
        FluidBox(FluidConfig(boundary=(("PERIODIC", "OUTFLOW"),) * 3))
    box = FluidBox(FluidConfig(n_cells=(8, 8, 8)))
    with pytest.raises(GfxError):
        box.step(-1.0)
