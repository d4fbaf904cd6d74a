"""A chart of several bricks on one device (gfx_fluid_chart_*) against one
brick of the whole chart: every step, every brick decomposition and boundary
mix, the conserved state of every proper cell and the CFL time step agree
bit for bit, and so do the face ghosts, the shock features seen across brick
faces and the boundary fluence on the chart's faces.  The single brick is
itself checked against the oracle (test_gpu_parity.py and the others), so
this pins the chart to the oracle too; one case checks it directly.

The reference (Chart_SLD__Form.f90:131-1097) exchanges the ghost layers of
faces and edges between bricks, clears the shock flags on the chart's
boundary only (FluidFeatures_P__Form.f90:313-336) and records the boundary
fluence on the chart's faces only (IncrementDivergence_FV__Form.f90:
1002-1069): a decomposition must not change any result.

The bit-level claims are the exact build's, so these tests pin it.  The fast
build lets the compiler fuse multiply-adds, and a brick's kernels may fuse
differently from the whole chart's; there the chart agrees with the single
brick to the last bits (the last test)."""
import numpy as np
import pytest

from genasis_b200 import problems
from genasis_b200.chart import FluidChart
from genasis_b200.config import FluidConfig
from genasis_b200.fluid import FluidBox
from tests.gpu_helpers import assert_parity, to_np

pytestmark = pytest.mark.gpu

P, O, R = "PERIODIC", "OUTFLOW", "REFLECTING"


def _cases():
    out = []
    cfg = FluidConfig(n_cells=(64, 64, 64), riemann_solver="HLLC", boundary=((P, P),) * 3,
                      courant_factor=0.8, n_ramp_cycles=1)
    out.append(("hllc_periodic_64_2x2x2", cfg, problems.random_state(cfg, seed=31), (2, 2, 2)))
    cfg = FluidConfig(n_cells=(64, 64, 64), riemann_solver="HLL", boundary=((O, O),) * 3,
                      courant_factor=0.8, n_ramp_cycles=1)
    out.append(("hll_outflow_64_2x2x2", cfg, problems.random_state(cfg, seed=32), (2, 2, 2)))
    cfg = FluidConfig(n_cells=(64, 64, 64), riemann_solver="HLLC",
                      boundary=((P, P), (R, O), (O, R)), courant_factor=0.8)
    out.append(("hllc_mixed_64_2x2x2", cfg, problems.random_state(cfg, seed=33), (2, 2, 2)))
    cfg = FluidConfig(n_cells=(48, 36, 40), riemann_solver="HLLC",
                      boundary=((R, R), (P, P), (O, O)), courant_factor=0.8)
    out.append(("hllc_ragged_3x2x5", cfg, problems.random_state(cfg, seed=34), (3, 2, 5)))
    cfg = FluidConfig(n_cells=(40, 24, 32), riemann_solver="HLLC",
                      boundary=((O, R), (R, O), (P, P)), courant_factor=0.8)
    out.append(("hllc_thin_bricks_10x6x1", cfg, problems.random_state(cfg, seed=35),
                (10, 6, 1)))
    cfg, prim = problems.rayleigh_taylor((16, 16, 32))
    out.append(("rt_gravity_reflecting_2x2x4", cfg, prim, (2, 2, 4)))
    cfg, prim = problems.kelvin_helmholtz(32)
    out.append(("kh_hllc_periodic_1x1x1", cfg, prim, (1, 1, 1)))
    cfg, prim = problems.kelvin_helmholtz(32)
    out.append(("kh_hllc_periodic_1x4x1", cfg, prim, (1, 4, 1)))
    return out


CASES = _cases()
IDS = [c[0] for c in CASES]


def _pair(cfg, prim, n_bricks):
    box = FluidBox(cfg, variant="exact")
    box.compute_from_primitive(prim)
    chart = FluidChart(cfg, n_bricks, variant="exact")
    chart.from_primitive(prim)
    return box, chart


def _face_ghosts(chart, b):
    """Index of brick b's values that are ghosts along exactly one axis."""
    g = 2
    n = [chart.brick_cells[d] for d in (2, 1, 0)]
    m = [k + 2 * g for k in n]
    z, y, x = np.meshgrid(*[np.arange(k) for k in m], indexing="ij")
    out = np.zeros(m, dtype=int)
    for t, k in zip((z, y, x), n):
        out += (t < g) | (t >= g + k)
    return out == 1


@pytest.mark.parametrize("name,cfg,prim,n_bricks", CASES, ids=IDS)
def test_chart_steps_equal_the_single_brick_bitwise(name, cfg, prim, n_bricks):
    box, chart = _pair(cfg, prim, n_bricks)
    p = cfg.proper
    for i in range(4):
        dt = box.compute_time_step(i)
        assert chart.compute_time_step(i) == dt, (name, i)
        box.step(dt)
        chart.step(dt)
        g, c = to_np(box.U), chart.gather()
        for f in range(6):
            assert np.array_equal(g[f][p], c[f][p]), "%s step %d field %d" % (name, i, f)
    # face ghosts: the images across brick faces, the boundary's ghosts on
    # the chart's faces, as the single brick holds them at those positions
    for b, u in enumerate(chart.U):
        mine = to_np(u)
        ref = g[(slice(None),) + chart._region(b)]
        sel = _face_ghosts(chart, b)
        for f in range(6):
            assert np.array_equal(mine[f][sel], ref[f][sel]), (name, "ghosts", b, f)
    box.close()
    chart.close()


@pytest.mark.parametrize("name,cfg,prim,n_bricks", CASES[:4], ids=IDS[:4])
def test_chart_evolve_equals_the_single_brick_evolve(name, cfg, prim, n_bricks):
    box, chart = _pair(cfg, prim, n_bricks)
    t_b, c_b = box.evolve(1e30, 0.0, 0, max_cycles=11)
    t_c, c_c = chart.evolve(1e30, 0.0, 0, max_cycles=11)
    assert (t_b, c_b) == (t_c, c_c)
    g, c = to_np(box.U), chart.gather()
    p = cfg.proper
    for f in range(6):
        assert np.array_equal(g[f][p], c[f][p]), (name, f)
    # and on from a state set from conserved values (features detected
    # across the brick faces from the conserved state)
    box.set_conserved(box.U.clone())
    box.detect_features()
    chart.set_conserved(g)
    dt = box.compute_time_step(11)
    box.step(dt)
    chart.step(dt)
    g, c = to_np(box.U), chart.gather()
    for f in range(6):
        assert np.array_equal(g[f][p], c[f][p]), (name, "after set_conserved", f)
    # the chart adds its bricks' sums: another order of the same terms
    tb, tc = box.totals(), chart.totals()
    assert np.allclose(tb, tc, rtol=0.0, atol=1e-13 * np.abs(tb).max()), (tb, tc)
    box.close()
    chart.close()


def _chart_fluence(chart, fl):
    """The chart's boundary fluence [6][6][chart face] assembled from the
    bricks' arrays (each brick records on the chart's faces only)."""
    N = [int(v) for v in chart.config.n_cells]
    n = chart.brick_cells
    fs = max(N[1] * N[2], N[0] * N[2], N[0] * N[1])
    out = np.zeros((6, 6, fs))
    # face -> (axis, side); a face's values are indexed a + na b over its
    # transverse cells: x faces (y, z), y faces (x, z), z faces (x, y)
    trans = {0: (1, 2), 1: (0, 2), 2: (0, 1)}
    for b, f in enumerate(fl):
        f = to_np(f)
        ib = chart.index[b]
        for face in range(6):
            a, side = divmod(face, 2)
            if ib[a] != (0 if side == 0 else chart.n_bricks[a] - 1):
                assert not f[:, face].any(), "brick %d records on an inner face" % b
                continue
            ta, tb = trans[a]
            for jb in range(n[tb]):
                for ja in range(n[ta]):
                    ga = ja + ib[ta] * n[ta]
                    gb = jb + ib[tb] * n[tb]
                    out[:, face, ga + N[ta] * gb] = f[:, face, ja + n[ta] * jb]
    return out


@pytest.mark.parametrize("name,cfg,prim,n_bricks", [CASES[2], CASES[3]], ids=[IDS[2], IDS[3]])
def test_chart_fluence_on_the_chart_faces_equals_the_single_brick(name, cfg, prim, n_bricks):
    box, chart = _pair(cfg, prim, n_bricks)
    fl_b = box.new_fluence()
    fl_c = chart.new_fluence()
    for i in range(2):
        dt = box.compute_time_step(i)
        box.step(dt, fl_b)
        chart.step(dt, fl_c)
    ref = to_np(fl_b)
    got = _chart_fluence(chart, fl_c)
    assert np.array_equal(got, ref[:, :, :got.shape[2]]), name
    box.close()
    chart.close()


def test_chart_matches_the_oracle_free_run():
    """The chart and the oracle from the same primitives, the oracle's time
    steps: D, S and G agree bit for bit after every step (DS to the parity
    bar: log and pow of CUDA and of the C library)."""
    from oracle.oracle import Oracle

    name, cfg, prim, n_bricks = CASES[2]
    chart = FluidChart(cfg, n_bricks, variant="exact")
    chart.from_primitive(prim)
    o = Oracle(cfg)
    o.set_primitive(prim)
    p = cfg.proper
    for i in range(3):
        dt = o.timestep(i)
        assert chart.compute_time_step(i) == dt, (name, i)
        o.step(dt)
        chart.step(dt)
        c, r = chart.gather(), o.conserved()
        assert_parity(c, r, cfg, "%s step %d" % (name, i))
        for f in range(5):
            assert np.array_equal(c[f][p], r[f][p]), (name, i, f)
    chart.close()


def test_chart_rejects_uneven_bricks_and_single_brick_calls():
    from genasis_b200 import lib

    cfg = FluidConfig(n_cells=(30, 16, 16))
    with pytest.raises(lib.GfxError):
        FluidChart(cfg, (4, 1, 1))  # 30 cells do not split into 4
    with pytest.raises(lib.GfxError):
        FluidChart(FluidConfig(n_cells=(12, 16, 16)), (4, 1, 1))  # 3 cells per brick
    chart = FluidChart(FluidConfig(n_cells=(16, 16, 16)), (2, 1, 1))
    import ctypes

    h = ctypes.c_void_p()
    chart.call("gfx_fluid_chart_brick", chart.h, 0, ctypes.byref(h), None)
    rc = lib.load().gfx_fluid_step(h, ctypes.c_void_p(chart.U[0].data_ptr()), 1e-3, None, None)
    assert rc == -1 and "chart" in lib.last_error()
    chart.close()


def test_chart_on_the_fast_build_stays_within_the_last_bits():
    from tests.gpu_helpers import quantity_errors

    name, cfg, prim, n_bricks = CASES[0]
    box = FluidBox(cfg, variant="fast")
    box.compute_from_primitive(prim)
    chart = FluidChart(cfg, n_bricks, variant="fast")
    chart.from_primitive(prim)
    for i in range(5):
        dt = box.compute_time_step(i)
        assert chart.compute_time_step(i) == pytest.approx(dt, rel=1e-14), (name, i)
        box.step(dt)
        chart.step(dt)
        q = quantity_errors(chart.gather(), box.U.detach().cpu().numpy(), cfg.proper)
        assert max(q) <= 1e-13, (name, i, q)
    box.close()
    chart.close()
