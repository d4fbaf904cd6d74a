"""CPU tests of the oracle (the reference restatement) and of the properties
of the reference step that the CUDA kernels rely on.

The reference ships no golden vectors for this path and cannot be compiled
here (Fortran + MPI), so the oracle is pinned by hand-derived known answers,
invariants of the scheme and the committed regression fixtures."""
import math

import numpy as np
import pytest

from genasis_b200 import problems
from genasis_b200.config import FluidConfig
from oracle.oracle import Oracle


def proper(cfg):
    return cfg.proper


def test_geometry_matches_python_restatement_bitwise():
    for n, lo, hi in [(16, 0.0, 1.0), (37, 0.0, 1.0), (384, 0.0, 0.5), (768, 0.0, 1.0)]:
        cfg = FluidConfig(n_cells=(n, 4, 4), min_coordinate=(lo, 0, 0), max_coordinate=(hi, 1, 1))
        o = Oracle(cfg)
        c, wl, wr = o.geometry(0)
        pc, pwl, pwr = problems.axis_geometry(n, lo, hi)
        assert np.array_equal(c, pc) and np.array_equal(wl, pwl) and np.array_equal(wr, pwr)


def test_ghost_widths_are_single_precision():
    # Chart_Template.f90 declares the ghost widths real(KDL): single precision.
    n = 768
    c, wl, wr = problems.axis_geometry(n, 0.0, 1.0)
    ghost_width = wl[0] + wr[0]
    proper_width = wl[2] + wr[2]
    assert ghost_width != proper_width
    assert abs(ghost_width - proper_width) < 1e-7 * proper_width
    assert float(np.float32(ghost_width)) == pytest.approx(ghost_width, rel=1e-15)


def _uniform(cfg, v=(0.3, -0.2, 0.1)):
    prim = np.zeros((5,) + cfg.shape)
    prim[0] = 1.3
    for d in range(3):
        prim[1 + d] = v[d]
    prim[4] = 2.0
    return prim


@pytest.mark.parametrize("rs", ["HLL", "HLLC"])
@pytest.mark.parametrize("bc", ["OUTFLOW", "PERIODIC"])
def test_uniform_state_has_zero_increment(rs, bc):
    cfg = FluidConfig(n_cells=(8, 6, 5), riemann_solver=rs, boundary=((bc, bc),) * 3)
    o = Oracle(cfg)
    o.set_primitive(_uniform(cfg, (0.0, 0.0, 0.0) if bc == "OUTFLOW" else (0.3, -0.2, 0.1)))
    K = o.increment(1e-3)
    assert np.all(K[(slice(None),) + cfg.proper] == 0.0)


def test_linear_profile_is_reconstructed_exactly():
    # A linear density with uniform velocity and pressure: the limiter returns
    # the profile's slope, the two face states agree, the HLL diffusion term
    # vanishes and K_D = -dt v dN/dx in the interior.
    n = 24
    cfg = FluidConfig(n_cells=(n, 4, 4), riemann_solver="HLL")
    X, Y, Z = problems.centers(cfg)
    prim = np.zeros((5,) + cfg.shape)
    slope = 0.5
    prim[0] = 1.0 + slope * X
    prim[1] = 1.0
    prim[4] = 2.5
    o = Oracle(cfg)
    o.set_primitive(prim)
    dt = 1e-3
    K = o.increment(dt)
    kd = K[0][cfg.proper][:, :, 3:-3]
    assert np.allclose(kd, -dt * slope, rtol=1e-10, atol=0)


@pytest.mark.parametrize("rs", ["HLL", "HLLC"])
def test_periodic_totals_are_conserved(rs):
    cfg, prim = problems.sine_wave(16, riemann_solver=rs)
    o = Oracle(cfg)
    o.set_primitive(prim)
    U0 = o.conserved()
    for i in range(4):
        o.step(o.timestep(i))
    U1 = o.conserved()
    p = cfg.proper
    for f in range(5):
        scale = np.abs(U0[f][p]).sum() + 1.0
        assert abs(U1[f][p].sum() - U0[f][p].sum()) <= 1e-13 * scale


def test_outflow_change_equals_boundary_fluence():
    cfg = FluidConfig(n_cells=(12, 10, 8), riemann_solver="HLLC")
    prim = problems.random_state(cfg, seed=3)
    o = Oracle(cfg)
    o.set_primitive(prim)
    p = cfg.proper
    # volume and face areas of the uniform interior cells
    w = [problems.axis_geometry(int(cfg.n_cells[d]), 0.0, 1.0)[1][2] * 2 for d in range(3)]
    vol = w[0] * w[1] * w[2]
    areas = [w[1] * w[2], w[2] * w[0], w[0] * w[1]]
    U0 = o.conserved()
    fl = o.new_fluence()
    o.step(o.timestep(5), fl)
    U1 = o.conserved()
    for f in range(5):
        dq = (U1[f][p].sum() - U0[f][p].sum()) * vol
        net = sum(areas[d] * (fl[f, 2 * d].sum() - fl[f, 2 * d + 1].sum()) for d in range(3))
        assert dq == pytest.approx(net, rel=1e-9, abs=1e-12)


def test_sod_keeps_transverse_symmetry():
    cfg, prim = problems.sod(16)
    o = Oracle(cfg)
    o.set_primitive(prim)
    for i in range(3):
        o.step(o.timestep(i))
    U = o.conserved()[(slice(None),) + cfg.proper]
    assert np.array_equal(U[0], U[0][:, ::-1, :])
    assert np.array_equal(U[0], U[0][::-1, :, :])
    assert np.all(U[2] == 0.0) and np.all(U[3] == 0.0)


def _exact_sod_density(x, t, gamma=1.4):
    """Exact solution of the Sod problem (Toro, ch. 4) at x (diaphragm 0.5)."""
    rl, pl, rr, pr = 1.0, 1.0, 0.125, 0.1
    cl, cr = math.sqrt(gamma * pl / rl), math.sqrt(gamma * pr / rr)

    def f(p, rk, pk, ck):
        if p > pk:
            A, B = 2 / ((gamma + 1) * rk), (gamma - 1) / (gamma + 1) * pk
            return (p - pk) * math.sqrt(A / (p + B))
        return 2 * ck / (gamma - 1) * ((p / pk) ** ((gamma - 1) / (2 * gamma)) - 1)

    lo, hi = 1e-6, 10.0
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if f(mid, rl, pl, cl) + f(mid, rr, pr, cr) > 0:
            hi = mid
        else:
            lo = mid
    ps = 0.5 * (lo + hi)
    us = 0.5 * (f(ps, rr, pr, cr) - f(ps, rl, pl, cl))
    rsl = rl * (ps / pl) ** (1 / gamma)
    rsr = rr * ((ps / pr + (gamma - 1) / (gamma + 1)) / ((gamma - 1) / (gamma + 1) * ps / pr + 1))
    shock = us * 0 + math.sqrt(gamma * pr / rr) * math.sqrt((gamma + 1) / (2 * gamma) * ps / pr
                                                             + (gamma - 1) / (2 * gamma))
    csl = cl * (ps / pl) ** ((gamma - 1) / (2 * gamma))
    out = np.empty_like(x)
    for i, xi in enumerate(x):
        s = (xi - 0.5) / t
        if s < -cl:
            out[i] = rl
        elif s < us - csl:
            u = 2 / (gamma + 1) * (cl + s)
            c = cl - (gamma - 1) / 2 * u
            out[i] = rl * (c / cl) ** (2 / (gamma - 1))
        elif s < us:
            out[i] = rsl
        elif s < shock:
            out[i] = rsr
        else:
            out[i] = rr
    return out


def test_sod_tracks_the_exact_riemann_solution():
    n = 96
    cfg = FluidConfig(n_cells=(n, 4, 4), riemann_solver="HLL", courant_factor=0.8,
                      n_ramp_cycles=1)
    prim = problems.riemann(cfg, 1.0, 1.0, (0, 0, 0), 0.125, 0.1, (0, 0, 0), (0.5, 0, 0),
                            (1.0, 0, 0))
    o = Oracle(cfg)
    o.set_primitive(prim)
    t, i = 0.0, 0
    while t < 0.15 - 1e-14:
        dt = min(o.timestep(i), 0.15 - t)
        o.step(dt)
        t += dt
        i += 1
    x = problems.axis_geometry(n, 0.0, 1.0)[0][2:-2]
    rho = o.conserved()[0][cfg.proper][2, 2, :]
    err = np.abs(rho - _exact_sod_density(x, t)).mean()
    assert err < 0.02


def compact_flags(P, V, n):
    """DIFFUSIVE_FLUX_I bits from the proper cells only, as the CUDA kernels
    compute them (valid for a single brick, see FluidFeatures_P__Kernel.f90)."""
    nz, ny, nx = n
    shock = np.zeros((3, nz, ny, nx), dtype=bool)
    for e in range(3):
        ax = 2 - e
        Pm = np.roll(P, 1, axis=ax)
        Vm = np.roll(V[e], 1, axis=ax)
        dP = np.abs(P - Pm)
        pmin = np.maximum(np.minimum(P, Pm), math.sqrt(np.finfo(float).tiny))
        s = (dP / pmin > 0.1) & (V[e] - Vm <= 0.0)
        idx = [slice(None)] * 3
        idx[ax] = 0
        s[tuple(idx)] = False
        shock[e] = s
    flags = np.zeros((3, nz, ny, nx), dtype=bool)
    for d in range(3):
        for e in range(3):
            if e == d:
                continue
            s = shock[e]
            ae, ad = 2 - e, 2 - d
            acc = s | np.roll(s, -1, axis=ae) | np.roll(s, 1, axis=ad) | np.roll(
                np.roll(s, -1, axis=ae), 1, axis=ad)
            flags[d] |= acc
    interior = np.zeros((nz, ny, nx), dtype=bool)
    interior[1:-1, 1:-1, 1:-1] = True
    return flags & interior[None]


@pytest.mark.parametrize("bc", ["OUTFLOW", "PERIODIC", "REFLECTING"])
def test_feature_flags_depend_on_proper_cells_only(bc):
    cfg = FluidConfig(n_cells=(14, 11, 9), boundary=((bc, bc),) * 3)
    o = Oracle(cfg)
    o.set_primitive(problems.random_state(cfg, seed=7))
    o.step(o.timestep(3))
    feat = o.features()
    aux = o.aux()
    prim = o.primitive()
    p = cfg.proper
    P = aux[0][p]
    V = [prim[1 + d][p] for d in range(3)]
    mine = compact_flags(P, V, P.shape)
    ref = np.stack([feat[d][p] > 0 for d in range(3)])
    assert ref.any()
    assert np.array_equal(mine, ref)
    # the outer face of each direction (a ghost index) never carries a flag
    g = cfg.n_ghost_layers
    for d in range(3):
        idx = list(cfg.proper)
        idx[2 - d] = g + int(cfg.n_cells[d])
        assert not feat[d][tuple(idx)].any()


@pytest.mark.parametrize("bc", ["OUTFLOW", "REFLECTING"])
def test_proper_results_do_not_depend_on_physical_ghosts(bc):
    cfg = FluidConfig(n_cells=(10, 9, 8), boundary=((bc, bc),) * 3, riemann_solver="HLLC")
    prim = problems.random_state(cfg, seed=11)
    a, b = Oracle(cfg), Oracle(cfg)
    a.set_primitive(prim)
    U = a.conserved()
    U2 = U.copy()
    ghost = np.ones(cfg.shape, dtype=bool)
    ghost[cfg.proper] = False
    rng = np.random.default_rng(0)
    U2[0][ghost] *= 1.0 + 0.5 * rng.uniform(size=ghost.sum())
    U2[4][ghost] *= 1.0 + 0.5 * rng.uniform(size=ghost.sum())
    a.set_conserved(U)
    b.set_conserved(U2)
    for i in range(2):
        dt = a.timestep(i)
        assert dt == b.timestep(i)
        a.step(dt)
        b.step(dt)
    p = (slice(None),) + cfg.proper
    assert np.array_equal(a.conserved()[p], b.conserved()[p])


def test_conserved_entropy_input_is_dead():
    # UseEntropy = .false.: ComputeFromConserved rewrites DS = N SB, so the
    # incoming DS (and its increment) never reach the next state.
    cfg = FluidConfig(n_cells=(9, 8, 7), riemann_solver="HLLC")
    o1, o2 = Oracle(cfg), Oracle(cfg)
    o1.set_primitive(problems.random_state(cfg, seed=5))
    U = o1.conserved()
    U2 = U.copy()
    U2[5] = np.random.default_rng(1).normal(size=U2[5].shape)
    o1.set_conserved(U)
    o2.set_conserved(U2)
    o1.step(1e-3)
    o2.step(1e-3)
    assert np.array_equal(o1.conserved(), o2.conserved())


def test_time_step_ramp():
    cfg, prim = problems.sod(8, n_ramp_cycles=10)
    o = Oracle(cfg)
    o.set_primitive(prim)
    full = o.timestep(50)
    assert o.timestep(0) == pytest.approx(0.1 * full, rel=1e-15)
    assert o.timestep(4) == pytest.approx(0.5 * full, rel=1e-15)
    tsi = o.inverse_timestep()
    assert full == cfg.courant_factor * (1.0 / tsi)


def test_time_step_of_a_uniform_flow():
    """ComputeTimeStepKernel_CSL (Integrator_C_PS__Kernel.f90:122-142) on a
    uniform state: the inverse CFL time is sum_d max(FEP_d, -FEM_d) / dX_d
    with FEP_d = V_d + CS, FEM_d = V_d - CS and CS = sqrt(gamma P / N), and the
    step is CourantFactor over it."""
    rho, p0, v = 1.3, 0.7, (0.4, -0.25, 0.0)
    n = (8, 10, 12)
    cfg = FluidConfig(n_cells=n, boundary=(("PERIODIC", "PERIODIC"),) * 3, courant_factor=0.8,
                      n_ramp_cycles=1)
    prim = np.zeros((5,) + cfg.shape)
    prim[0] = rho
    for d in range(3):
        prim[1 + d] = v[d]
    prim[4] = p0 / (cfg.adiabatic_index - 1.0)
    o = Oracle(cfg)
    o.set_primitive(prim)
    cs = math.sqrt(cfg.adiabatic_index * p0 / rho)
    tsi = sum(max(v[d] + cs, -(v[d] - cs)) * n[d] for d in range(3))
    assert o.inverse_timestep() == pytest.approx(tsi, rel=1e-13)
    assert o.timestep(0) == pytest.approx(0.8 / tsi, rel=1e-13)


# ---- PARABOLIC reconstruction (IncrementDivergence_FV__Kernel.f90:296-596) ----

def test_parabolic_reconstructs_a_linear_profile_exactly():
    n = 24
    cfg = FluidConfig(n_cells=(n, 4, 4), riemann_solver="HLL", reconstruction="PARABOLIC")
    X, Y, Z = problems.centers(cfg)
    prim = np.zeros((5,) + cfg.shape)
    prim[0] = 1.0 + 0.5 * X
    prim[1] = 1.0
    prim[4] = 2.5
    o = Oracle(cfg)
    o.set_primitive(prim)
    dt = 1e-3
    K = o.increment(dt)
    kd = K[0][cfg.proper][:, :, 3:-3]
    assert np.allclose(kd, -dt * 0.5, rtol=1e-9, atol=0)


@pytest.mark.parametrize("rs", ["HLL", "HLLC"])
def test_parabolic_periodic_totals_are_conserved(rs):
    cfg, prim = problems.sine_wave(16, riemann_solver=rs)
    cfg.reconstruction = "PARABOLIC"
    o = Oracle(cfg)
    o.set_primitive(prim)
    U0 = o.conserved()
    for i in range(4):
        o.step(o.timestep(i))
    U1 = o.conserved()
    p = cfg.proper
    for f in range(5):
        scale = np.abs(U0[f][p]).sum() + 1.0
        assert abs(U1[f][p].sum() - U0[f][p].sum()) <= 1e-13 * scale


def test_parabolic_is_more_accurate_than_linear_on_the_sine_wave():
    errs = {}
    for rec in ("LINEAR", "PARABOLIC"):
        cfg, prim = problems.sine_wave(24)
        cfg.reconstruction = rec
        o = Oracle(cfg)
        o.set_primitive(prim)
        t, i = 0.0, 0
        while t < 0.1:
            dt = o.timestep(i)
            o.step(dt)
            t += dt
            i += 1
        errs[rec] = problems.l1_error(o.primitive()[0], problems.sine_density(cfg, t), cfg)
    assert errs["PARABOLIC"] < 0.8 * errs["LINEAR"], errs


def test_parabolic_keeps_sod_close_to_the_exact_solution():
    n = 96
    cfg = FluidConfig(n_cells=(n, 4, 4), riemann_solver="HLL", courant_factor=0.8,
                      n_ramp_cycles=1, reconstruction="PARABOLIC")
    prim = problems.riemann(cfg, 1.0, 1.0, (0, 0, 0), 0.125, 0.1, (0, 0, 0), (0.5, 0, 0),
                            (1.0, 0, 0))
    o = Oracle(cfg)
    o.set_primitive(prim)
    t, i = 0.0, 0
    while t < 0.15 - 1e-14:
        dt = min(o.timestep(i), 0.15 - t)
        o.step(dt)
        t += dt
        i += 1
    x = problems.axis_geometry(n, 0.0, 1.0)[0][2:-2]
    rho = o.conserved()[0][cfg.proper][2, 2, :]
    assert np.abs(rho - _exact_sod_density(x, t)).mean() < 0.02


@pytest.mark.parametrize("rs", ["HLLC", "HLL"])
def test_hllc_keeps_a_stationary_contact_and_hll_spreads_it(rs):
    """A density jump at rest under a uniform pressure (a contact).  HLLC's
    centre wave is the contact itself: the centre speed AC = SN / MD is 0
    exactly (SN = p_L - p_R = 0), so every face carries (0, p, 0, 0, 0) and
    the steps leave D, S and G unchanged bit for bit (no shock flags arise:
    the pressure is uniform).  HLL has no centre wave: its mass flux at the
    jump, -AP AM (D_R - D_L) / (AP + AM), spreads the contact."""
    cfg = FluidConfig(n_cells=(16, 6, 6), boundary=(("OUTFLOW", "OUTFLOW"),) * 3,
                      riemann_solver=rs, courant_factor=0.8, n_ramp_cycles=1)
    prim = problems.riemann(cfg, 1.0, 1.0, (0.0, 0.0, 0.0), 0.5, 1.0, (0.0, 0.0, 0.0),
                            (0.5, 0.0, 0.0), (1.0, 0.0, 0.0))
    o = Oracle(cfg)
    o.set_primitive(prim)
    p = (slice(0, 5),) + cfg.proper
    U0 = o.conserved()[p].copy()
    if rs == "HLLC":
        for i in range(3):
            o.step(o.timestep(i))
        assert np.array_equal(o.conserved()[p], U0)
        assert not o.features().any()
    else:
        o.step(o.timestep(0))
        changed = np.argwhere(o.conserved()[p][0] != U0[0])
        # the jump lies between x cells 7 and 8; each of the two stages
        # carries the change one cell further on either side
        assert sorted(set(int(x) for x in changed[:, 2])) == [6, 7, 8, 9]


@pytest.mark.parametrize("axis", [1, 2])
def test_sod_along_each_axis_is_the_same_tube(axis):
    """The Sod tube along y or z, relabelled (axes and momentum components
    swapped), is the tube along x: the three directions run one code path.
    Along y it is the same bit for bit.  Along z it agrees to a few ulps: the
    cell volume is the product of the widths in axis order, (w0 w1) w2
    (GeometryFlat_Kernel.f90:22-41), and the widths of the repeated-addition
    edges differ by ulps from cell to cell, so relabelling x and z
    re-associates the product (x and y only swap its first, commutative,
    pair); so does the reference's x, y, z order of adding the directions'
    round-off-sized transverse terms (HLLC next to HLL faces of the shock
    flags)."""
    def run(d):
        cfg = FluidConfig(n_cells=(12, 12, 12), boundary=(("OUTFLOW", "OUTFLOW"),) * 3,
                          riemann_solver="HLLC", courant_factor=0.8, n_ramp_cycles=1)
        point, normal = [0.0, 0.0, 0.0], [0.0, 0.0, 0.0]
        point[d], normal[d] = 0.5, 1.0
        prim = problems.riemann(cfg, 1.0, 1.0, (0.0, 0.0, 0.0), 0.125, 0.1, (0.0, 0.0, 0.0),
                                point, normal)
        o = Oracle(cfg)
        o.set_primitive(prim)
        for i in range(4):
            o.step(o.timestep(i))
        return o.conserved()

    Ux, Ud = run(0), run(axis)
    # arrays are [field][z][y][x]: array axis 3 - d holds direction d
    swapped = np.swapaxes(Ud, 3, 3 - axis)
    perm = [0, 1, 2, 3, 4, 5]
    perm[1], perm[1 + axis] = perm[1 + axis], perm[1]
    if axis == 1:
        assert np.array_equal(swapped[perm], Ux)
    else:
        assert float(np.abs(swapped[perm] - Ux).max()) <= 1e-14 * float(np.abs(Ux).max())


@pytest.mark.parametrize("rs", ["HLL", "HLLC"])
def test_reflecting_walls_keep_the_mass_in(rs):
    """A box with reflecting walls on all six faces.  The ghost cells mirror
    the wall cells with the normal velocity reversed.  The reference rounds
    the ghost widths through single precision (real(KDL)), so where the width
    survives that (1/8 along z) the reconstructed face states at a wall are
    exact mirrors, the outer wave speeds come out equal and the mass flux
    through the wall is exactly zero; where it does not (1/10, 1/9) the
    mirrored slopes differ in their last bits and a round-off-sized mass flux
    crosses.  The total mass changes by round-off only."""
    cfg = FluidConfig(n_cells=(10, 9, 8), boundary=(("REFLECTING", "REFLECTING"),) * 3,
                      riemann_solver=rs, courant_factor=0.8, n_ramp_cycles=1)
    prim = problems.random_state(cfg, seed=5)
    o = Oracle(cfg)
    o.set_primitive(prim)
    p = cfg.proper
    m0 = o.conserved()[0][p].sum()
    for i in range(3):
        fl = o.new_fluence()  # [field][face: x in, x out, y in, y out, z in, z out][...]
        o.step(o.timestep(i), fl)
        assert not fl[0, 4:].any()
        assert float(np.abs(fl[0, :4]).max()) <= 1e-10
    m1 = o.conserved()[0][p].sum()
    assert abs(m1 - m0) <= 1e-13 * m0


def test_gravity_source_on_a_uniform_gas_at_rest():
    """A uniform gas at rest under the uniform acceleration a along z
    (ApplyGravity_F, ApplyGravity_F__Command.f90:124-264, with the gradient
    (0, 0, a)): every flux divergence vanishes, so one RK2 step is the source
    alone.  Stage 1 gives K_S3 = -N a dt and no energy term (V = 0); stage 2,
    on Y with V3 = -a dt, gives K_S3 = -N a dt again and K_G = -N (V3 a) dt.
    So S3 = -N a dt and G = G0 + N a^2 dt^2 / 2: the work of gravity is the
    kinetic energy gained."""
    a, rho, p0 = 0.1, 1.5, 1.0
    cfg = FluidConfig(n_cells=(8, 8, 8), boundary=(("PERIODIC", "PERIODIC"),) * 3,
                      riemann_solver="HLLC", courant_factor=0.8, n_ramp_cycles=1,
                      uniform_acceleration=a)
    prim = np.zeros((5,) + cfg.shape)
    prim[0] = rho
    prim[4] = p0 / (cfg.adiabatic_index - 1.0)
    o = Oracle(cfg)
    o.set_primitive(prim)
    p = (slice(None),) + cfg.proper
    U0 = o.conserved()[p].copy()
    dt = o.timestep(0)
    o.step(dt)
    U1 = o.conserved()[p]
    assert np.array_equal(U1[0], U0[0])
    assert np.all(U1[1] == 0.0) and np.all(U1[2] == 0.0)
    assert np.allclose(U1[3], -rho * a * dt, rtol=1e-14, atol=0.0)
    assert np.allclose(U1[4] - U0[4], 0.5 * rho * a * a * dt * dt, rtol=1e-9, atol=0.0)
