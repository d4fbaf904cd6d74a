"""ctypes binding of libgfx_fluid.so (the C ABI of include/gfx_fluid.h).

The library is the only compute path: if it is missing or cannot load, every
entry point raises; there is no CPU fallback.

Two builds of the same C ABI exist (genasis_b200/build_ext.py): "exact"
(libgfx_fluid.so, the reference's rounding) and "fast"
(libgfx_fluid_fast.so, fused multiply-adds and products with reciprocals,
within 1e-12 per step of the exact one).  Every call names its variant;
without one it takes GFX_FLUID_VARIANT from the environment, else "exact".
A handle belongs to the library that created it."""
import ctypes
import os

from .config import GfxConfig

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_FILES = {"exact": "libgfx_fluid.so", "fast": "libgfx_fluid_fast.so"}
LIB_PATH = os.path.join(_HERE, LIB_FILES["exact"])

GFX_OK = 0
STATUS = {
    -1: "GFX_ERR_ARGUMENT",
    -2: "GFX_ERR_CUDA",
    -3: "GFX_ERR_UNSUPPORTED",
    -4: "GFX_ERR_STATE",
    -5: "GFX_ERR_TIMEOUT",
    -6: "GFX_ERR_NO_MEMORY",
}

# name -> (restype, argtypes); every entry point returns an int status.
P = ctypes.c_void_p
D = ctypes.c_double
I = ctypes.c_int
SZ = ctypes.c_size_t
SIGNATURES = {
    "gfx_fluid_config_default": [ctypes.POINTER(GfxConfig)],
    "gfx_fluid_create": [ctypes.POINTER(GfxConfig), ctypes.POINTER(P)],
    "gfx_fluid_destroy": [P],
    "gfx_fluid_n_values": [P, ctypes.POINTER(SZ)],
    "gfx_fluid_geometry": [P, I, P, P, P],
    "gfx_fluid_from_primitive": [P, P, P, P],
    "gfx_fluid_to_primitive": [P, P, P, P, P],
    "gfx_fluid_detect_features": [P, P, P],
    "gfx_fluid_clear_features": [P, P],
    "gfx_fluid_get_features": [P, P, P],
    "gfx_fluid_increment": [P, P, P, D, D, P, P],
    "gfx_fluid_fluence_face_size": [P, ctypes.POINTER(SZ)],
    "gfx_fluid_step": [P, P, D, P, P],
    "gfx_fluid_step_sources": [P, P, D, P, P, P],
    "gfx_fluid_step_host": [P, P, D, P],
    "gfx_fluid_timestep": [P, P, I, ctypes.POINTER(D), P],
    "gfx_fluid_evolve": [P, P, D, I, D, I, ctypes.POINTER(D), ctypes.POINTER(I), P],
    "gfx_fluid_evolve_timed": [P, P, D, I, D, I, ctypes.POINTER(D), ctypes.POINTER(I),
                               ctypes.POINTER(D), P],
    "gfx_fluid_step_timed": [P, P, D, P, P, P],
    "gfx_fluid_kernel_launches": [P, ctypes.POINTER(ctypes.c_longlong)],
    "gfx_fluid_batch_create": [I, P, P, ctypes.POINTER(P)],
    "gfx_fluid_batch_destroy": [P],
    "gfx_fluid_batch_set_clocks": [P, D, I],
    "gfx_fluid_batch_evolve": [P, D, I, P],
    "gfx_fluid_batch_clocks": [P, P, P, P],
    "gfx_fluid_batch_kernel_launches": [P, ctypes.POINTER(ctypes.c_longlong)],
    "gfx_fluid_step_adjoint": [P, P, D, P, P, P, I, P],
    "gfx_fluid_step_noalloc": [ctypes.POINTER(GfxConfig), P, D, I, P, P],
    "gfx_fluid_step_branches": [P, P, D, I, P, P],
    "gfx_fluid_check_state": [P, P, P],
    "gfx_fluid_set_tuning": [P, I, I, I],
    "gfx_fluid_totals": [P, P, P, P],
    "gfx_fluid_resume": [P, P],
    "gfx_fluid_chart_create": [ctypes.POINTER(GfxConfig), ctypes.POINTER(I), ctypes.POINTER(P)],
    "gfx_fluid_chart_destroy": [P],
    "gfx_fluid_chart_n_bricks": [P, ctypes.POINTER(I)],
    "gfx_fluid_chart_brick": [P, I, ctypes.POINTER(P), ctypes.POINTER(I)],
    "gfx_fluid_chart_bind": [P, P],
    "gfx_fluid_chart_from_primitive": [P, P, P],
    "gfx_fluid_chart_set_conserved": [P, P],
    "gfx_fluid_chart_timestep": [P, I, ctypes.POINTER(D), P],
    "gfx_fluid_chart_step": [P, D, P, P],
    "gfx_fluid_chart_evolve": [P, D, I, D, I, ctypes.POINTER(D), ctypes.POINTER(I), P],
    "gfx_fluid_chart_kernel_launches": [P, ctypes.POINTER(ctypes.c_longlong)],
    "gfx_fluid_last_error": [ctypes.c_char_p, SZ],
    "gfx_fluid_debug_fail_allocation": [I],
}

_libs = {}


class GfxError(RuntimeError):
    def __init__(self, status, where, message):
        super().__init__("%s: %s (%s)" % (where, message, STATUS.get(status, status)))
        self.status = status


def default_variant():
    v = os.environ.get("GFX_FLUID_VARIANT", "exact")
    if v not in LIB_FILES:
        raise ValueError("GFX_FLUID_VARIANT=%r: expected one of %s" % (v, sorted(LIB_FILES)))
    return v


def lib_path(variant=None):
    return os.path.join(_HERE, LIB_FILES[variant or default_variant()])


def load(variant=None):
    """Loads the in-tree library of the variant (raises if it is absent)."""
    variant = variant or default_variant()
    if variant in _libs:
        return _libs[variant]
    path = lib_path(variant)
    if not os.path.exists(path):
        raise RuntimeError(
            "%s is not built (run genasis_b200/build_ext.py or __graft_entry__.build()); "
            "there is no fallback path" % os.path.basename(path))
    lib = ctypes.CDLL(path)
    for name, args in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = ctypes.c_int
        fn.argtypes = args
    _libs[variant] = lib
    return lib


def last_error(variant=None):
    buf = ctypes.create_string_buffer(1024)
    load(variant).gfx_fluid_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def call(name, *args, variant=None):
    """Calls an entry point of the variant's library and raises GfxError on
    a nonzero status."""
    rc = getattr(load(variant), name)(*args)
    if rc != GFX_OK:
        raise GfxError(rc, name, last_error(variant))
    return rc


def exported_symbols():
    return list(SIGNATURES)
