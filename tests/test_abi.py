"""The C ABI library loads and exports every entry point that
include/gfx_fluid.h declares (no compute calls without a GPU)."""
import ctypes
import os
import re

import pytest

from genasis_b200 import lib
from genasis_b200.config import FluidConfig, GfxConfig

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    text = open(os.path.join(ROOT, "include", "gfx_fluid.h")).read()
    return sorted(set(re.findall(r"\bint\s+(gfx_fluid_\w+)\s*\(", text)))


def test_library_is_built_for_sm100a():
    from genasis_b200 import build_ext

    path = build_ext.build()
    assert os.path.exists(path)
    assert "arch=compute_100a,code=sm_100a" in " ".join(build_ext.NVCC_FLAGS)
    assert "--fmad=false" in build_ext.NVCC_FLAGS


def test_every_declared_symbol_is_exported_and_bound():
    so = ctypes.CDLL(lib.LIB_PATH)
    names = header_functions()
    assert len(names) >= 15
    for n in names:
        assert hasattr(so, n), n
    assert set(names) == set(lib.exported_symbols())


def test_config_struct_layout_matches_header_defaults():
    c = GfxConfig()
    lib.call("gfx_fluid_config_default", ctypes.byref(c))
    ref = FluidConfig().to_c()
    assert c.n_ghost_layers == 2
    assert c.riemann_solver == 1  # HLLC (Fluid_ASC__Form.f90:128-137)
    assert c.limiter_parameter == 1.4 and c.adiabatic_index == 1.4
    assert c.shock_threshold == 0.1 and c.courant_factor == 0.7
    assert c.n_ramp_cycles == 100 and c.use_limiter == 1
    assert ctypes.sizeof(c) == ctypes.sizeof(ref)


def _cuda():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:  # noqa: BLE001
        return False


@pytest.mark.skipif(_cuda(), reason="checks the no-device error path")
def test_create_reports_an_error_without_a_device():
    c = FluidConfig(n_cells=(8, 8, 8)).to_c()
    h = ctypes.c_void_p()
    rc = lib.load().gfx_fluid_create(ctypes.byref(c), ctypes.byref(h))
    assert rc != 0
    assert lib.last_error()


def test_invalid_configs_are_rejected_before_any_device_call():
    for cfg in [FluidConfig(n_cells=(3, 8, 8)),
                FluidConfig(n_ghost_layers=3),
                FluidConfig(boundary=(("PERIODIC", "OUTFLOW"),) * 3),
                FluidConfig(n_ramp_cycles=0)]:
        c = cfg.to_c()
        h = ctypes.c_void_p()
        rc = lib.load().gfx_fluid_create(ctypes.byref(c), ctypes.byref(h))
        assert rc in (-1, -3), rc
        assert "n_" in lib.last_error() or "PERIODIC" in lib.last_error()
