"""Initial conditions of the benchmark problems, as primitive fields
[N, V1, V2, V3, E] over every value of the brick (ghosts included), the way
the reference's problem set-ups fill the Current before ComputeFromPrimitive.

  sod / riemann   RiemannProblem_Form.f90:111-136 (states), :237-275 (diaphragm
                  test <= 1e-10 on the plane's signed distance)
  sine_wave       plane-wave advection of PlaneWave_Template.f90 with the
                  density profile 1 + 0.5 sin(2 pi (x + y + z)), v = (1, 1, 1), p = 1
  kelvin_helmholtz, rayleigh_taylor (RayleighTaylor_Form.f90:83-104, 246-279)
  random_bricks   independent bricks with seeded two-state Riemann problems
All inputs are seeded synthetic data with the benchmark's shapes.
"""
import math

import numpy as np

from .config import FluidConfig


def axis_geometry(n, xmin, xmax, g=2):
    """Cell centres and half widths of one axis over the ghost-inclusive range,
    as Chart_Template.f90:478-560 builds them: edges by repeated addition of
    (max - min) / n, ghost widths rounded through single precision (the
    reference declares them real(KDL)), centres 0.5 (E_i + E_i+1)."""
    m = n + 2 * g
    edge = [0.0] * (m + 1)
    off = g - 1  # edge[off + i] = Edge(i)
    width = (xmax - xmin) / float(n)
    edge[off + 1] = float(xmin)
    for i in range(2, n + 2):
        edge[off + i] = edge[off + i - 1] + width
    for ic in range(1, g + 1):
        w_ig = float(np.float32(edge[off + ic + 1] - edge[off + ic]))
        w_og = float(np.float32(edge[off + n - ic + 2] - edge[off + n - ic + 1]))
        edge[off + 1 - ic] = edge[off + 2 - ic] - w_ig
        edge[off + n + 1 + ic] = edge[off + n + ic] + w_og
    c = np.array([0.5 * (edge[t] + edge[t + 1]) for t in range(m)])
    wl = np.array([c[t] - edge[t] for t in range(m)])
    wr = np.array([edge[t + 1] - c[t] for t in range(m)])
    return c, wl, wr


def centers(cfg):
    """(X, Y, Z) broadcastable over the (z, y, x) ghost-inclusive shape."""
    xs = [axis_geometry(int(cfg.n_cells[d]), cfg.min_coordinate[d], cfg.max_coordinate[d],
                        cfg.n_ghost_layers)[0] for d in range(3)]
    return xs[0][None, None, :], xs[1][None, :, None], xs[2][:, None, None]


def _prim(cfg):
    return np.zeros((5,) + cfg.shape)


def riemann(cfg, rho_l, p_l, v_l, rho_r, p_r, v_r, point, normal):
    """Two-state Riemann problem: the left state where
    normal . (x - point) <= 1e-10 (RiemannProblem_Form.f90:251-272)."""
    X, Y, Z = centers(cfg)
    gm1 = cfg.adiabatic_index - 1.0
    side = (normal[0] * (X - point[0]) + normal[1] * (Y - point[1])
            + normal[2] * (Z - point[2])) <= 1.0e-10
    prim = _prim(cfg)
    prim[0] = np.where(side, rho_l, rho_r)
    for d in range(3):
        prim[1 + d] = np.where(side, v_l[d], v_r[d])
    prim[4] = np.where(side, p_l / gm1, p_r / gm1)
    return prim


def sod(n=128, riemann_solver="HLL", courant=0.8, n_ramp_cycles=1):
    """3-D Sod tube along x on the unit cube, outflow on all faces."""
    cfg = FluidConfig(n_cells=(n, n, n), boundary=(("OUTFLOW", "OUTFLOW"),) * 3,
                      riemann_solver=riemann_solver, courant_factor=courant,
                      n_ramp_cycles=n_ramp_cycles)
    prim = riemann(cfg, 1.0, 1.0, (0.0, 0.0, 0.0), 0.125, 0.1, (0.0, 0.0, 0.0),
                   (0.5, 0.0, 0.0), (1.0, 0.0, 0.0))
    return cfg, prim


def sine_density(cfg, t=0.0, velocity=(1.0, 1.0, 1.0)):
    X, Y, Z = centers(cfg)
    return 1.0 + 0.5 * np.sin(2.0 * math.pi * ((X - velocity[0] * t) + (Y - velocity[1] * t)
                                               + (Z - velocity[2] * t)))


def sine_wave(n=256, riemann_solver="HLLC", courant=0.8, n_ramp_cycles=1):
    """Density wave advected along the diagonal of the periodic unit cube."""
    cfg = FluidConfig(n_cells=(n, n, n), boundary=(("PERIODIC", "PERIODIC"),) * 3,
                      riemann_solver=riemann_solver, courant_factor=courant,
                      n_ramp_cycles=n_ramp_cycles)
    prim = _prim(cfg)
    prim[0] = sine_density(cfg)
    prim[1:4] = 1.0
    prim[4] = 1.0 / (cfg.adiabatic_index - 1.0)
    return cfg, prim


def l1_error(density, exact, cfg):
    """PlaneWave_Template.f90:106-113: sum |N - N_exact| / sum |N_exact| over
    proper cells."""
    p = cfg.proper
    d = np.asarray(density)[p]
    e = np.asarray(exact)[p]
    return float(np.abs(d - e).sum() / np.abs(e).sum())


def kelvin_helmholtz(n=128, seed=20261204, riemann_solver="HLLC", courant=0.8,
                     n_ramp_cycles=1):
    cfg = FluidConfig(n_cells=(n, n, n), boundary=(("PERIODIC", "PERIODIC"),) * 3,
                      riemann_solver=riemann_solver, courant_factor=courant,
                      n_ramp_cycles=n_ramp_cycles)
    X, Y, Z = centers(cfg)
    inside = np.abs(Y - 0.5) < 0.25
    shape = cfg.shape
    prim = _prim(cfg)
    prim[0] = np.broadcast_to(np.where(inside, 2.0, 1.0), shape)
    prim[1] = np.broadcast_to(np.where(inside, 0.5, -0.5), shape)
    rng = np.random.default_rng(seed)
    noise = rng.uniform(-1.0, 1.0, size=shape)
    prim[2] = 0.01 * np.sin(4.0 * math.pi * X) + 1.0e-3 * noise
    prim[3] = 0.0
    prim[4] = 2.5 / (cfg.adiabatic_index - 1.0)
    return cfg, prim


def rayleigh_taylor(shape=(384, 384, 768), seed=20261206, g=0.1, riemann_solver="HLLC",
                    courant=0.8, n_ramp_cycles=1):
    nx, ny, nz = shape
    cfg = FluidConfig(n_cells=(nx, ny, nz), max_coordinate=(0.5, 0.5, 1.0),
                      boundary=(("PERIODIC", "PERIODIC"), ("PERIODIC", "PERIODIC"),
                                ("REFLECTING", "REFLECTING")),
                      riemann_solver=riemann_solver, courant_factor=courant,
                      n_ramp_cycles=n_ramp_cycles, uniform_acceleration=g)
    X, Y, Z = centers(cfg)
    rho = np.where(Z > 0.5, 2.0, 1.0)
    p = 2.5 - rho * g * (Z - 0.5)
    prim = _prim(cfg)
    full = cfg.shape
    prim[0] = np.broadcast_to(rho, full)
    rng = np.random.default_rng(seed)
    window = np.abs(Z - 0.5) < 0.1
    mode = 0.01 * (1.0 + np.cos(4.0 * math.pi * X)) * (1.0 + np.cos(4.0 * math.pi * Y)) / 4.0
    prim[3] = np.where(window, mode, 0.0) + 1.0e-3 * rng.uniform(-1.0, 1.0, size=full)
    prim[4] = np.broadcast_to(p / (cfg.adiabatic_index - 1.0), full)
    return cfg, prim


def random_bricks(count=512, seed=20261203, lo=16, hi=96, riemann_solver="HLL",
                  courant=0.8, n_ramp_cycles=1, only=None):
    """Independent bricks with seeded sizes and two-state Riemann problems:
    per-axis edges U{lo..hi}; (rho, p) log-uniform in [0.1, 10]; velocity
    components U[-1, 1]; a diaphragm through a uniform point of the unit cube
    with a normal uniform on the sphere.  only: the indices whose primitive
    arrays are built (the others come as (config, None)); the draws are the
    same whatever it holds, so a rank of a sharded run gets its bricks exactly
    as the whole set has them."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = tuple(int(v) for v in rng.integers(lo, hi + 1, size=3))
        cfg = FluidConfig(n_cells=n, boundary=(("OUTFLOW", "OUTFLOW"),) * 3,
                          riemann_solver=riemann_solver, courant_factor=courant,
                          n_ramp_cycles=n_ramp_cycles)
        rho_l, p_l, rho_r, p_r = np.exp(rng.uniform(math.log(0.1), math.log(10.0), size=4))
        v_l = rng.uniform(-1.0, 1.0, size=3)
        v_r = rng.uniform(-1.0, 1.0, size=3)
        point = rng.uniform(0.0, 1.0, size=3)
        normal = rng.normal(size=3)
        normal = normal / np.linalg.norm(normal)
        prim = None
        if only is None or i in only:
            prim = riemann(cfg, rho_l, p_l, v_l, rho_r, p_r, v_r, point, normal)
        out.append((cfg, prim))
    return out


def random_state(cfg, seed=1, shocks=True):
    """A rough random state for parity tests: smooth background plus jumps."""
    rng = np.random.default_rng(seed)
    X, Y, Z = centers(cfg)
    shape = cfg.shape
    prim = _prim(cfg)
    prim[0] = 1.0 + 0.3 * np.sin(2 * math.pi * X) * np.cos(2 * math.pi * Y) + 0.2 * Z
    prim[1] = 0.3 * np.sin(2 * math.pi * Y)
    prim[2] = -0.2 * np.cos(2 * math.pi * Z)
    prim[3] = 0.1 * np.sin(2 * math.pi * X)
    prim[4] = 2.0 + 0.5 * np.cos(2 * math.pi * (X + Z))
    prim = np.broadcast_to(prim, (5,) + shape).copy()
    prim += 0.05 * rng.uniform(-1, 1, size=prim.shape) * np.array([1, 1, 1, 1, 1])[:, None, None, None]
    if shocks:
        left = (X + 0.3 * Y) < 0.45
        prim[0] = np.where(left, prim[0] * 4.0, prim[0])
        prim[4] = np.where(left, prim[4] * 8.0, prim[4])
        prim[1] = np.where(left, prim[1] + 0.8, prim[1])
    return prim


def noisy(prim, amp=2e-2, seed=7):
    """prim with seeded relative noise of amplitude amp on N and E and
    absolute noise on V: a state without exactly uniform fields, where the
    limiter and the wave-speed maxima are differentiable (gradient checks)."""
    rng = np.random.default_rng(seed)
    out = np.array(prim, dtype=np.float64, copy=True)
    out[0] *= 1.0 + amp * rng.uniform(-1.0, 1.0, size=out[0].shape)
    out[4] *= 1.0 + amp * rng.uniform(-1.0, 1.0, size=out[4].shape)
    for d in range(1, 4):
        out[d] += amp * rng.uniform(-1.0, 1.0, size=out[d].shape)
    return out
