"""Shock detection at the threshold: states whose pressure jumps put
|dP| / min(P) within a few ulps of the shock threshold, on a ragged brick
that several detection tiles and z chunks cover.  The DIFFUSIVE_FLUX_I flags
of the CUDA path (from the primitives kept at initialisation, from the
conserved state, and inside an evolve from the primitives stage 2 stored)
equal the oracle's, and so do the states they steer."""
import numpy as np
import pytest

from genasis_b200.config import FluidConfig
from tests.gpu_helpers import assert_parity, make_pair, to_np

pytestmark = pytest.mark.gpu


def band_state(cfg, seed, near_fraction=0.08):
    """Pressure base * (1 + thr (1 + delta)) on the cells of odd i + j + k and
    base elsewhere: delta = m 2^-52 (|m| <= 16) on a random few cells, -1/2 on
    the rest (no shock).  The velocities fall along every axis, so the
    velocity condition of a shock holds everywhere."""
    rng = np.random.default_rng(seed)
    shape = cfg.shape
    k, j, i = np.meshgrid(*(np.arange(s) for s in shape), indexing="ij")
    thr = cfg.shock_threshold
    near = rng.random(shape) < near_fraction
    delta = np.where(near, rng.integers(-16, 17, size=shape) * 2.0**-52, -0.5)
    base = 0.7
    P = np.where((i + j + k) % 2 == 1, base * (1.0 + thr * (1.0 + delta)), base)
    prim = np.zeros((5,) + shape)
    prim[0] = 1.0 + 0.25 * rng.random(shape)
    prim[1] = -0.01 * i
    prim[2] = -0.013 * j
    prim[3] = -0.017 * k
    prim[4] = P / (cfg.adiabatic_index - 1.0)
    return prim


def _cfg():
    return FluidConfig(n_cells=(37, 19, 70), riemann_solver="HLLC", courant_factor=0.4,
                       n_ramp_cycles=1)


def test_band_is_exercised():
    """The designed quotients straddle the threshold within 2^-50 of it."""
    cfg = _cfg()
    prim = band_state(cfg, seed=3)
    P = prim[4] * (cfg.adiabatic_index - 1.0)
    q = np.abs(np.diff(P, axis=2)) / np.minimum(P[:, :, 1:], P[:, :, :-1])
    rel = q / cfg.shock_threshold - 1.0
    assert np.count_nonzero(np.abs(rel) < 2.0**-50) > 50
    assert np.count_nonzero((np.abs(rel) > 2.0**-50) & (np.abs(rel) < 2.0**-47)) > 50


def _flags_agree(box, o, cfg):
    f = to_np(box.features())
    ref = o.features()
    p = cfg.proper
    for d in range(3):
        assert np.array_equal(((f >> d) & 1)[p] > 0, ref[d][p] > 0), d
    return int(np.count_nonzero(f[p]))


@pytest.mark.parametrize("seed", [3, 4])
def test_flags_at_the_threshold_match_oracle(seed):
    cfg = _cfg()
    box, o = make_pair(cfg, band_state(cfg, seed))
    # from the primitives kept at initialisation
    box.detect_features()
    o.detect_features()
    n0 = _flags_agree(box, o, cfg)
    assert 0 < n0 < cfg.n_proper
    # from the conserved state after a step
    for i in range(2):
        dt = o.timestep(i)
        o.step(dt)
        box.step(dt)
    assert_parity(to_np(box.U), o.conserved(), cfg, "band step")
    box.detect_features()
    o.detect_features()
    _flags_agree(box, o, cfg)
    box.close()


def test_evolve_at_the_threshold_matches_oracle_loop():
    """Inside an evolve the detection reads the primitives stage 2 stored."""
    cfg = _cfg()
    box, o = make_pair(cfg, band_state(cfg, seed=5))
    t, c = box.evolve(1.0, 0.0, 0, max_cycles=4)
    assert c == 4
    tt = 0.0
    for i in range(4):
        dt = o.timestep(i)
        o.step(dt)
        tt += dt
    assert t == pytest.approx(tt, rel=1e-15)
    assert_parity(to_np(box.U), o.conserved(), cfg, "band evolve")
    box.close()
