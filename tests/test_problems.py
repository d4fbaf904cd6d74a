"""The benchmark inputs as the benchmark defines them, checked at small sizes
against genasis_b200.problems: the periodic sine wave (C2), the Sod tube
(C1), Kelvin-Helmholtz (C4), Rayleigh-Taylor (C5) and the random bricks (C3),
with their boundaries, solvers, seeds and value distributions.  Each expected
field is written out here from the definition, not from the generator."""
import math

import numpy as np
import pytest

from genasis_b200 import problems

GAMMA = 1.4


def _grid(cfg):
    X, Y, Z = problems.centers(cfg)
    shape = cfg.shape
    return (np.broadcast_to(X, shape), np.broadcast_to(Y, shape), np.broadcast_to(Z, shape))


def _bcs(cfg):
    return tuple(tuple(side.upper() for side in axis) for axis in cfg.boundary)


def test_sine_wave_is_the_periodic_density_wave():
    cfg, prim = problems.sine_wave(12)
    assert tuple(cfg.n_cells) == (12, 12, 12)
    assert _bcs(cfg) == (("PERIODIC", "PERIODIC"),) * 3
    assert cfg.riemann_solver.upper() == "HLLC" and cfg.courant_factor == 0.8
    X, Y, Z = _grid(cfg)
    assert np.array_equal(prim[0], 1.0 + 0.5 * np.sin(2.0 * math.pi * (X + Y + Z)))
    assert np.all(prim[1:4] == 1.0)
    assert np.all(prim[4] == 1.0 / (GAMMA - 1.0))  # p = 1
    # cell centres of the unit cube
    p = cfg.proper
    assert X[p].min() == pytest.approx(0.5 / 12) and X[p].max() == pytest.approx(1 - 0.5 / 12)


def test_sod_tube_has_its_two_states_about_x_one_half():
    cfg, prim = problems.sod(16)
    assert _bcs(cfg) == (("OUTFLOW", "OUTFLOW"),) * 3
    assert cfg.riemann_solver.upper() == "HLL"
    X, _, _ = _grid(cfg)
    left = X <= 0.5 + 1e-10
    assert np.all(prim[0][left] == 1.0) and np.all(prim[0][~left] == 0.125)
    assert np.all(prim[4][left] == 1.0 / (GAMMA - 1.0))
    assert np.all(prim[4][~left] == 0.1 / (GAMMA - 1.0))
    assert np.all(prim[1:4] == 0.0)


def test_kelvin_helmholtz_layers_and_seeded_perturbation():
    cfg, prim = problems.kelvin_helmholtz(16)
    assert _bcs(cfg) == (("PERIODIC", "PERIODIC"),) * 3
    assert cfg.riemann_solver.upper() == "HLLC"
    X, Y, _ = _grid(cfg)
    inside = np.abs(Y - 0.5) < 0.25
    assert np.array_equal(prim[0], np.where(inside, 2.0, 1.0))
    assert np.array_equal(prim[1], np.where(inside, 0.5, -0.5))
    # vy = 0.01 sin(4 pi x) + 1e-3 U[-1, 1], seed 20261204, cells in x-fastest order
    u = np.random.default_rng(20261204).uniform(-1.0, 1.0, size=cfg.shape)
    assert np.array_equal(prim[2], 0.01 * np.sin(4.0 * math.pi * X) + 1.0e-3 * u)
    assert np.all(prim[3] == 0.0)
    assert np.all(prim[4] == 2.5 / (GAMMA - 1.0))


def test_rayleigh_taylor_column_is_hydrostatic_with_a_seeded_mode():
    g = 0.1
    cfg, prim = problems.rayleigh_taylor(shape=(8, 8, 16))
    assert _bcs(cfg) == (("PERIODIC", "PERIODIC"), ("PERIODIC", "PERIODIC"),
                         ("REFLECTING", "REFLECTING"))
    assert cfg.uniform_acceleration == g and cfg.riemann_solver.upper() == "HLLC"
    assert tuple(cfg.max_coordinate) == (0.5, 0.5, 1.0)
    widths = [(cfg.max_coordinate[d] - cfg.min_coordinate[d]) / cfg.n_cells[d] for d in range(3)]
    assert widths[0] == widths[1] == widths[2]  # cubic cells
    X, Y, Z = _grid(cfg)
    rho = np.where(Z > 0.5, 2.0, 1.0)
    assert np.array_equal(prim[0], rho)
    assert np.array_equal(prim[4], (2.5 - rho * g * (Z - 0.5)) / (GAMMA - 1.0))
    assert np.all(prim[1] == 0.0) and np.all(prim[2] == 0.0)
    u = np.random.default_rng(20261206).uniform(-1.0, 1.0, size=cfg.shape)
    mode = 0.01 * (1.0 + np.cos(4.0 * math.pi * X)) * (1.0 + np.cos(4.0 * math.pi * Y)) / 4.0
    assert np.array_equal(prim[3], np.where(np.abs(Z - 0.5) < 0.1, mode, 0.0) + 1.0e-3 * u)


def test_random_bricks_follow_the_seeded_draws():
    bricks = problems.random_bricks(count=6)
    rng = np.random.default_rng(20261203)
    for cfg, prim in bricks:
        # draw order per brick: edges (nx, ny, nz) in U{16..96}, then the
        # states (rho_l, p_l, rho_r, p_r log-uniform in [0.1, 10]), the two
        # velocities U[-1, 1]^3, the diaphragm point, its normal
        n = tuple(int(v) for v in rng.integers(16, 97, size=3))
        assert tuple(cfg.n_cells) == n
        rho_l, p_l, rho_r, p_r = np.exp(rng.uniform(math.log(0.1), math.log(10.0), size=4))
        v_l, v_r = rng.uniform(-1.0, 1.0, size=3), rng.uniform(-1.0, 1.0, size=3)
        point = rng.uniform(0.0, 1.0, size=3)
        normal = rng.normal(size=3)
        normal = normal / np.linalg.norm(normal)
        assert _bcs(cfg) == (("OUTFLOW", "OUTFLOW"),) * 3
        assert cfg.riemann_solver.upper() == "HLL" and cfg.courant_factor == 0.8
        X, Y, Z = _grid(cfg)
        left = (normal[0] * (X - point[0]) + normal[1] * (Y - point[1])
                + normal[2] * (Z - point[2])) <= 1.0e-10
        assert np.array_equal(prim[0], np.where(left, rho_l, rho_r))
        assert np.array_equal(prim[4], np.where(left, p_l, p_r) / (GAMMA - 1.0))
        for d in range(3):
            assert np.array_equal(prim[1 + d], np.where(left, v_l[d], v_r[d]))
        assert 0.1 <= min(rho_l, rho_r) and max(rho_l, rho_r) <= 10.0


def test_l1_error_is_the_plane_wave_norm_over_proper_cells():
    """sum |N - N_exact| / sum |N_exact| over the proper cells only: ghost
    values do not enter; the exact profile is the initial one translated by
    v t."""
    cfg, prim = problems.sine_wave(8)
    exact = problems.sine_density(cfg, t=0.25)
    rho = exact.copy()
    p = cfg.proper
    rho[p] += 1e-3
    ghost = np.ones(cfg.shape, dtype=bool)
    ghost[p] = False
    rho[ghost] += 7.0  # ghosts are left out of the norm
    expected = 1e-3 * rho[p].size / np.abs(exact[p]).sum()
    assert problems.l1_error(rho, exact, cfg) == pytest.approx(expected, rel=1e-12)
    X, Y, Z = _grid(cfg)
    shifted = 1.0 + 0.5 * np.sin(2.0 * math.pi * ((X - 0.25) + (Y - 0.25) + (Z - 0.25)))
    assert np.array_equal(exact, shifted)
