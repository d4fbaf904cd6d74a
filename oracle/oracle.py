"""ctypes wrapper of the CPU oracle (libgfx_oracle.so).

Test infrastructure only: tests/, the smoke check and bench.py's CPU legs use
it as the checker.  The genasis_b200 package never imports this module.

Parity status: unpinned by reference-run outputs (the Fortran reference cannot
be compiled here and ships no golden vectors); see fluid_oracle.c.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libgfx_oracle.so")
_lib = None

BC = {"OUTFLOW": 0, "REFLECTING": 1, "PERIODIC": 2}
RIEMANN = {"HLL": 0, "HLLC": 1}
RECONSTRUCTION = {"LINEAR": 0, "PARABOLIC": 1}


class OraConfig(ctypes.Structure):
    _fields_ = [
        ("n_cells", ctypes.c_int * 3),
        ("n_ghost_layers", ctypes.c_int),
        ("min_coordinate", ctypes.c_double * 3),
        ("max_coordinate", ctypes.c_double * 3),
        ("boundary", (ctypes.c_int * 2) * 3),
        ("riemann_solver", ctypes.c_int),
        ("use_limiter", ctypes.c_int),
        ("limiter_parameter", ctypes.c_double),
        ("adiabatic_index", ctypes.c_double),
        ("shock_threshold", ctypes.c_double),
        ("courant_factor", ctypes.c_double),
        ("baryon_density_min", ctypes.c_double),
        ("uniform_acceleration", ctypes.c_double),
        ("n_ramp_cycles", ctypes.c_int),
        ("reconstruction", ctypes.c_int),
    ]


def build():
    """Compile the oracle with its Makefile (gcc, -ffp-contract=off)."""
    subprocess.check_call(["make", "-s", "-C", _HERE], stdout=subprocess.DEVNULL)


def _load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        build()
    lib = ctypes.CDLL(_LIB_PATH)
    P = ctypes.c_void_p
    D = ctypes.c_double
    lib.ora_create.restype = P
    lib.ora_create.argtypes = [ctypes.POINTER(OraConfig)]
    lib.ora_destroy.argtypes = [P]
    lib.ora_n_values.restype = ctypes.c_size_t
    lib.ora_n_values.argtypes = [P]
    lib.ora_fluence_face_size.restype = ctypes.c_size_t
    lib.ora_fluence_face_size.argtypes = [P]
    lib.ora_geometry.argtypes = [P, ctypes.c_int, P, P, P]
    for name in ("ora_set_primitive", "ora_set_conserved", "ora_get_conserved",
                 "ora_get_primitive", "ora_get_aux", "ora_get_features",
                 "ora_set_features"):
        getattr(lib, name).argtypes = [P, P]
    lib.ora_clear_features.argtypes = [P]
    lib.ora_detect_features.argtypes = [P]
    lib.ora_increment.argtypes = [P, P, D, D, P]
    lib.ora_step.argtypes = [P, D, P]
    lib.ora_step_sources.argtypes = [P, D, P, P]
    lib.ora_timestep.restype = D
    lib.ora_timestep.argtypes = [P, ctypes.c_int]
    lib.ora_inverse_timestep.restype = D
    lib.ora_inverse_timestep.argtypes = [P]
    lib.ora_n_threads.restype = ctypes.c_int
    _lib = lib
    return lib


def make_config(cfg):
    """Fill the C struct from any object with the reference parameter fields
    (n_cells, min_coordinate, max_coordinate, boundary, riemann_solver, ...)."""
    c = OraConfig()
    for d in range(3):
        c.n_cells[d] = int(cfg.n_cells[d])
        c.min_coordinate[d] = float(cfg.min_coordinate[d])
        c.max_coordinate[d] = float(cfg.max_coordinate[d])
        for s in range(2):
            b = cfg.boundary[d][s]
            c.boundary[d][s] = BC[b] if isinstance(b, str) else int(b)
    c.n_ghost_layers = int(cfg.n_ghost_layers)
    rs = cfg.riemann_solver
    c.riemann_solver = RIEMANN[rs] if isinstance(rs, str) else int(rs)
    c.use_limiter = int(bool(cfg.use_limiter))
    c.limiter_parameter = float(cfg.limiter_parameter)
    c.adiabatic_index = float(cfg.adiabatic_index)
    c.shock_threshold = float(cfg.shock_threshold)
    c.courant_factor = float(cfg.courant_factor)
    c.baryon_density_min = float(cfg.baryon_density_min)
    c.uniform_acceleration = float(cfg.uniform_acceleration)
    c.n_ramp_cycles = int(cfg.n_ramp_cycles)
    rc = getattr(cfg, "reconstruction", "LINEAR")
    c.reconstruction = RECONSTRUCTION[rc] if isinstance(rc, str) else int(rc)
    return c


def _ptr(a):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(ctypes.c_void_p)


class Oracle:
    """One single-brick Fluid_P_I state with the reference's RK2 step.

    Arrays are numpy float64 in the reference layout [field][z][y][x] with
    n_ghost_layers ghosts on every side."""

    def __init__(self, cfg):
        self.lib = _load()
        self.cfg = cfg
        self._c = make_config(cfg)
        self.h = self.lib.ora_create(ctypes.byref(self._c))
        g = int(cfg.n_ghost_layers)
        self.shape = tuple(int(cfg.n_cells[2 - d]) + 2 * g for d in range(3))
        self.nV = int(self.lib.ora_n_values(self.h))
        self.face_size = int(self.lib.ora_fluence_face_size(self.h))

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.ora_destroy(self.h)
            self.h = None

    def geometry(self, axis):
        m = int(self.cfg.n_cells[axis]) + 2 * int(self.cfg.n_ghost_layers)
        c, wl, wr = (np.zeros(m) for _ in range(3))
        self.lib.ora_geometry(self.h, axis, _ptr(c), _ptr(wl), _ptr(wr))
        return c, wl, wr

    def set_primitive(self, prim):
        prim = np.ascontiguousarray(prim, dtype=np.float64)
        assert prim.shape == (5,) + self.shape
        self.lib.ora_set_primitive(self.h, _ptr(prim))

    def set_conserved(self, cons):
        cons = np.ascontiguousarray(cons, dtype=np.float64)
        assert cons.shape == (6,) + self.shape
        self.lib.ora_set_conserved(self.h, _ptr(cons))

    def conserved(self):
        out = np.zeros((6,) + self.shape)
        self.lib.ora_get_conserved(self.h, _ptr(out))
        return out

    def primitive(self):
        out = np.zeros((5,) + self.shape)
        self.lib.ora_get_primitive(self.h, _ptr(out))
        return out

    def aux(self):
        out = np.zeros((9,) + self.shape)
        self.lib.ora_get_aux(self.h, _ptr(out))
        return out

    def features(self):
        out = np.zeros((7,) + self.shape)
        self.lib.ora_get_features(self.h, _ptr(out))
        return out

    def set_features(self, feat):
        feat = np.ascontiguousarray(feat, dtype=np.float64)
        self.lib.ora_set_features(self.h, _ptr(feat))

    def clear_features(self):
        self.lib.ora_clear_features(self.h)

    def detect_features(self):
        self.lib.ora_detect_features(self.h)

    def increment(self, dt, weight_rk=1.0, K=None, fluence=None):
        if K is None:
            K = np.zeros((6,) + self.shape)
        fl = _ptr(fluence) if fluence is not None else None
        self.lib.ora_increment(self.h, _ptr(K), float(dt), float(weight_rk), fl)
        return K

    def new_fluence(self):
        return np.zeros((6, 6, self.face_size))

    def step(self, dt, fluence=None):
        fl = _ptr(fluence) if fluence is not None else None
        self.lib.ora_step(self.h, float(dt), fl)

    def step_sources(self, dt, fluence=None):
        """One step; returns its Sources records [10][nV]: the divergence
        sources of the six conserved fields, Gravitational_G, Gravitational_S_D."""
        fl = _ptr(fluence) if fluence is not None else None
        src = np.zeros((10, self.nV))
        self.lib.ora_step_sources(self.h, float(dt), fl, _ptr(src))
        return src

    def timestep(self, i_cycle):
        return float(self.lib.ora_timestep(self.h, int(i_cycle)))

    def inverse_timestep(self):
        return float(self.lib.ora_inverse_timestep(self.h))

    @staticmethod
    def n_threads():
        return int(_load().ora_n_threads())
