"""The oracle's Sources records of a step (ApplyDivergence_C /
RecordDivergenceKernel and ApplyGravity_F of the reference's Step_RK_C_ASC):
the records leave the step itself unchanged, the divergence records are zero
on ghosts, and over one step the records add up to the change of the state,
(U^{n+1} - U^n) / dt = S_divergence + S_gravitational, up to round-off."""
import numpy as np
import pytest

from genasis_b200 import problems
from genasis_b200.config import FluidConfig
from oracle.oracle import Oracle


def _cases():
    out = []
    cfg, prim = problems.rayleigh_taylor((8, 8, 16))
    out.append(("rt_gravity", cfg, prim))
    cfg = FluidConfig(n_cells=(11, 7, 9), riemann_solver="HLLC",
                      boundary=(("PERIODIC", "PERIODIC"), ("REFLECTING", "OUTFLOW"),
                                ("OUTFLOW", "OUTFLOW")))
    out.append(("random_hllc_mixed", cfg, problems.random_state(cfg, seed=11)))
    cfg = FluidConfig(n_cells=(9, 10, 8), riemann_solver="HLL", uniform_acceleration=-0.3)
    out.append(("random_hll_gravity", cfg, problems.random_state(cfg, seed=12, shocks=False)))
    return out


CASES = _cases()
IDS = [c[0] for c in CASES]


def _pair(cfg, prim):
    a, b = Oracle(cfg), Oracle(cfg)
    a.set_primitive(prim)
    b.set_primitive(prim)
    return a, b


@pytest.mark.parametrize("name,cfg,prim", CASES, ids=IDS)
def test_records_leave_the_step_unchanged(name, cfg, prim):
    a, b = _pair(cfg, prim)
    for i in range(2):
        dt = a.timestep(i)
        fa, fb = a.new_fluence(), b.new_fluence()
        a.step(dt, fa)
        b.step_sources(dt, fb)
        assert np.array_equal(a.conserved(), b.conserved()), (name, i)
        assert np.array_equal(fa, fb), (name, i)
        assert np.array_equal(a.features(), b.features()), (name, i)


@pytest.mark.parametrize("name,cfg,prim", CASES, ids=IDS)
def test_records_add_up_to_the_change_of_the_state(name, cfg, prim):
    o = Oracle(cfg)
    o.set_primitive(prim)
    shape = (10,) + tuple(cfg.shape)
    for i in range(2):
        dt = o.timestep(i)
        u0 = o.conserved()
        src = o.step_sources(dt).reshape(shape)
        u1 = o.conserved()
        # divergence records: zero on every ghost value
        ghost = np.ones(cfg.shape, dtype=bool)
        ghost[cfg.proper] = False
        assert not np.any(src[:6][:, ghost]), name
        grav = cfg.uniform_acceleration != 0.0
        if not grav:
            assert not np.any(src[6:]), name
        else:
            # no gradient along x and y: Gravitational_S_D 1, 2 are zero
            assert not np.any(src[7:9]), name
            assert np.all(src[9][cfg.proper] * np.sign(cfg.uniform_acceleration) < 0), name
        rate = (u1 - u0) / dt
        total = src[:5].copy()
        total[1:4] += src[7:10]
        total[4] += src[6]
        for f in range(5):
            scale = np.abs(u0[f][cfg.proper]).max() / dt
            err = np.abs(rate[f][cfg.proper] - total[f][cfg.proper]).max()
            assert err <= 1e-12 * scale, (name, i, f, err, scale)
