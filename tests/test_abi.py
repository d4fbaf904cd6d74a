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
    # the exact build rounds every operation on its own; the speed build fuses
    assert "--fmad=false" in build_ext.VARIANTS["exact"][1]
    assert "--fmad=true" in build_ext.VARIANTS["fast"][1]
    assert "-DGFX_FAST_MATH=1" in build_ext.VARIANTS["fast"][1]
    for v in ("exact", "fast"):
        assert os.path.exists(build_ext.lib_path(v)), v


@pytest.mark.parametrize("variant", ["exact", "fast"])
def test_every_declared_symbol_is_exported_and_bound(variant):
    so = ctypes.CDLL(lib.lib_path(variant))
    names = header_functions()
    assert len(names) >= 15
    for n in names:
        assert hasattr(so, n), n
    assert set(names) == set(lib.exported_symbols())


def test_fp64_probe_exports_and_refuses_bad_arguments():
    """libgfx_probe.so, the bench's FP64 rate probe, is built beside the
    library and checks its arguments before any CUDA call."""
    from genasis_b200 import build_ext

    build_ext.build()
    so = ctypes.CDLL(os.path.join(ROOT, "genasis_b200", "libgfx_probe.so"))
    f, ms = ctypes.c_double(), ctypes.c_double()
    fn = so.gfx_probe_fp64_chains
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                   ctypes.POINTER(ctypes.c_double)]
    assert fn(0, 4096, ctypes.byref(f), ctypes.byref(ms)) == -1
    assert fn(1, 0, ctypes.byref(f), ctypes.byref(ms)) == -1
    assert fn(1, (1 << 22) + 1, ctypes.byref(f), ctypes.byref(ms)) == -1
    assert fn(1, 4096, None, ctypes.byref(ms)) == -1
    assert hasattr(so, "gfx_probe_fp64")


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


def header_arg_counts():
    """Arguments of every declared entry point (a void list counts 0)."""
    text = open(os.path.join(ROOT, "include", "gfx_fluid.h")).read()
    out = {}
    for name, args in re.findall(r"\bint\s+(gfx_fluid_\w+)\s*\(([^)]*)\)", text):
        args = args.strip()
        out[name] = 0 if args in ("", "void") else args.count(",") + 1
    return out


def fortran_interfaces():
    """bind(c) name -> argument count of include/gfx_fluid_f.f90's interfaces."""
    text = open(os.path.join(ROOT, "include", "gfx_fluid_f.f90")).read()
    text = re.sub(r"&\s*\n\s*", " ", text)  # join continuation lines
    out = {}
    for args, name in re.findall(
            r"function\s+\w+\s*\(([^)]*)\)\s*bind\s*\(\s*c\s*,\s*name\s*=\s*'(\w+)'", text):
        out[name] = len([a for a in args.split(",") if a.strip()])
    return out


def test_fortran_binding_matches_the_header():
    h = header_arg_counts()
    f = fortran_interfaces()
    assert set(f) == set(h), set(f) ^ set(h)
    for name, n in h.items():
        assert f[name] == n, (name, f[name], n)


def test_fortran_config_type_has_the_c_layout():
    """Offsets of GFX_FluidConfig's components under the C alignment rules
    (which bind(c) types follow) equal those of the C struct."""
    text = open(os.path.join(ROOT, "include", "gfx_fluid_f.f90")).read()
    body = text.split("type, bind ( c ), public :: GFX_FluidConfig")[1].split("end type")[0]
    size = {"c_int": 4, "c_double": 8}
    off, offsets = 0, []
    fields = re.findall(r"(?:integer|real) \( (c_int|c_double) \) :: (\w+)(?: \(([^)]*)\))?", body)
    for kind, name, dims in fields:
        n = 1
        for d in (dims.split(",") if dims else []):
            n *= int(d)
        a = size[kind]
        off = (off + a - 1) // a * a
        offsets.append(off)
        off += a * n
    c_fields = [f[0] for f in GfxConfig._fields_]
    assert len(fields) == len(c_fields)
    assert offsets == [getattr(GfxConfig, f).offset for f in c_fields]


def _calls(text, name):
    """Argument lists (top-level comma count + 1) of every call to name."""
    out = []
    for m in re.finditer(r"\b%s\s*\(" % name, text):
        i, depth, args, nonempty = m.end(), 1, 1, False
        while depth:
            c = text[i]
            if c == "(":
                depth += 1
            elif c == ")":
                depth -= 1
            elif c == "," and depth == 1:
                args += 1
            elif not c.isspace() and c != "&":
                nonempty = True
            i += 1
        out.append(args if nonempty else 0)
    return out


def test_genasis_wrapper_calls_match_the_header():
    """include/gfx_fluid_genasis.f90 (the GenASiS-side wrapper) calls each C
    function with the header's number of arguments."""
    text = open(os.path.join(ROOT, "include", "gfx_fluid_genasis.f90")).read()
    text = "\n".join(l.split("!")[0] for l in text.splitlines())  # drop comments
    text = re.sub(r"&\s*\n\s*", " ", text)  # join continuation lines
    h = header_arg_counts()
    used = 0
    for name, n in h.items():
        for got in _calls(text, name):
            assert got == n, (name, got, n)
            used += 1
    assert used >= 6
