"""gfx_fluid_step_noalloc: the RK2 step for callers that cannot allocate
device memory (a host program whose memory manager has claimed the GPU's
memory into its own pool, or a code path that cannot take the device-wide
synchronisation of cudaMalloc / cudaFree).  It runs the step of
gfx_fluid_step without a handle, its buffers carved from a fixed array inside
the library, so its results must be those of the handle's step.

Two calls in a row on each case: the second call finds the array holding the
first call's contents and must still agree.  The file is named to be
collected last, so that a run stopping at the first failure has run every
other test before it."""
import ctypes

import numpy as np
import pytest

from genasis_b200 import lib, problems
from genasis_b200.config import FluidConfig
from tests.gpu_helpers import PARITY_RTOL, assert_parity, to_np

pytestmark = pytest.mark.gpu


def _torch():
    import torch

    return torch


def _p(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def _stream():
    return ctypes.c_void_p(_torch().cuda.current_stream().cuda_stream)


def _cases():
    rnd = FluidConfig(n_cells=(21, 13, 17), riemann_solver="HLLC",
                      boundary=(("OUTFLOW", "REFLECTING"), ("PERIODIC", "PERIODIC"),
                                ("REFLECTING", "OUTFLOW")))
    grav = FluidConfig(n_cells=(12, 10, 30), riemann_solver="HLL",
                       boundary=(("PERIODIC", "PERIODIC"), ("PERIODIC", "PERIODIC"),
                                 ("REFLECTING", "REFLECTING")),
                       uniform_acceleration=-0.1)
    sine_cfg, sine_prim = problems.sine_wave(37)  # the largest cube that fits
    return [
        ("random_hllc_mixed_bc", rnd, problems.random_state(rnd, seed=5)),
        ("random_hll_gravity", grav, problems.random_state(grav, seed=6)),
        ("sine_hllc_periodic_37", sine_cfg, sine_prim),
    ]


CASES = _cases()


@pytest.mark.parametrize("detect_first", [False, True], ids=["zero_features_first",
                                                           "features_from_the_first_step"])
@pytest.mark.parametrize("name,cfg,prim", CASES, ids=[c[0] for c in CASES])
def test_noalloc_step_matches_the_handle_step_twice(name, cfg, prim, detect_first):
    _run_pair(name, cfg, prim, detect_first, device="cuda")


def test_noalloc_step_on_a_second_device():
    """Each device holds its own copy of the array and its own launch set-up:
    the step on device 1 must agree with the handle's step there."""
    torch = _torch()
    if torch.cuda.device_count() < 2:
        pytest.skip("one CUDA device visible")
    name, cfg, prim = CASES[0]
    with torch.cuda.device(1):
        _run_pair(name + " on device 1", cfg, prim, True, device="cuda:1")


def _run_pair(name, cfg, prim, detect_first, device):
    torch = _torch()
    c = cfg.to_c()
    h = ctypes.c_void_p()
    lib.call("gfx_fluid_create", ctypes.byref(c), ctypes.byref(h))
    try:
        fs = ctypes.c_size_t()
        lib.call("gfx_fluid_fluence_face_size", h, ctypes.byref(fs))
        prim_d = torch.tensor(prim, dtype=torch.float64, device=device)
        U_ref = torch.zeros((6,) + cfg.shape, dtype=torch.float64, device=device)
        s = _stream()
        lib.call("gfx_fluid_from_primitive", h, _p(prim_d), _p(U_ref), s)
        # state from conserved values, as the no-allocation step takes it
        lib.call("gfx_fluid_to_primitive", h, _p(U_ref), None, None, s)
        U_na = U_ref.clone()
        fl_ref = torch.zeros((6, 6, fs.value), dtype=torch.float64, device="cuda")
        fl_na = torch.full_like(fl_ref, 7.0)  # stale values: the call must clear them
        for call in range(2):
            dt = ctypes.c_double()
            lib.call("gfx_fluid_timestep", h, _p(U_ref), call, ctypes.byref(dt), s)
            # the first step after initialisation runs on zero features, every
            # later one detects them from its input state; with detect_first
            # the handle detects them before its first step too
            if call == 0 and detect_first:
                lib.call("gfx_fluid_detect_features", h, _p(U_ref), s)
            lib.call("gfx_fluid_step", h, _p(U_ref), dt.value, _p(fl_ref), s)
            lib.call("gfx_fluid_step_noalloc", ctypes.byref(c), _p(U_na), dt.value,
                     1 if (call > 0 or detect_first) else 0, _p(fl_na), s)
            torch.cuda.synchronize()
            a, b = to_np(U_na), to_np(U_ref)
            everything = (slice(None),) * 3
            assert_parity(a, b, cfg, "%s call %d (all values)" % (name, call + 1),
                          rtol=PARITY_RTOL, index=everything)
            fa, fb = to_np(fl_na), to_np(fl_ref)
            scale = max(float(np.abs(fb).max()), 1e-300)
            assert float(np.abs(fa - fb).max()) <= PARITY_RTOL * scale, \
                "%s call %d fluence" % (name, call + 1)
    finally:
        lib.load().gfx_fluid_destroy(h)


def test_noalloc_step_rejects_bricks_beyond_its_scratch():
    torch = _torch()
    cfg = FluidConfig(n_cells=(38, 38, 38))
    c = cfg.to_c()
    U = torch.zeros((6,) + cfg.shape, dtype=torch.float64, device="cuda")
    rc = lib.load().gfx_fluid_step_noalloc(ctypes.byref(c), _p(U), 1e-3, 0, None, _stream())
    assert rc == -1  # GFX_ERR_ARGUMENT
    msg = lib.last_error()
    assert "no-allocation step has 4194304" in msg and "38 x 38 x 38" in msg
    assert float(to_np(U).max()) == 0.0  # rejected before any work
