"""Host-side mirror of the reference's operator interface for the fluid step.

The classes keep the reference's names and call surfaces, backed by the C ABI
of libgfx_fluid.so; PyTorch provides device memory and the current stream.

  FluidBox                 FluidBox_Form (Universes/FluidBox_Form.f90:37-241):
                           one brick, its Fluid_P_I current (the conserved state
                           U with ghosts) and features
  Step_RK2_C_ASC.compute   Step_RK_C_ASC_Template % Compute (time, time_step)
  IncrementDivergence_FV.compute
                           IncrementDivergence_FV_Form % Compute
                           (increment, time_step, weight_rk)
  Integrator_C_PS          ComputeTimeStep / Evolve of the integrator

Errors come back as GfxError (the library never aborts); the reference shows
them and calls PROGRAM_HEADER % Abort, which the caller may still do.
"""
import ctypes

import numpy as np

from . import lib
from .config import FluidConfig

# Fields of the Sources records (GFX_N_SOURCES of the C header)
N_SOURCES = 10


def _torch():
    import torch  # noqa: WPS433 (device memory and streams only)

    return torch


def _stream():
    return ctypes.c_void_p(_torch().cuda.current_stream().cuda_stream)


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


class FluidBox:
    """One brick of Fluid_P_I on the current CUDA device."""

    def __init__(self, config: FluidConfig, device=None, variant=None):
        torch = _torch()
        if not torch.cuda.is_available():
            raise RuntimeError("FluidBox needs a CUDA device (there is no CPU path)")
        self.config = config
        self.device = torch.device(device) if device is not None else torch.device("cuda")
        # the library build ("exact" or "fast", genasis_b200.lib) of this brick
        self.variant = variant or lib.default_variant()
        self._c = config.to_c()
        h = ctypes.c_void_p()
        self.call("gfx_fluid_create", ctypes.byref(self._c), ctypes.byref(h))
        self.h = h
        n = ctypes.c_size_t()
        self.call("gfx_fluid_n_values", self.h, ctypes.byref(n))
        self.n_values = int(n.value)
        fs = ctypes.c_size_t()
        self.call("gfx_fluid_fluence_face_size", self.h, ctypes.byref(fs))
        self.face_size = int(fs.value)
        self.U = torch.zeros((6,) + config.shape, dtype=torch.float64, device=self.device)

    def call(self, name, *args):
        """An entry point of this brick's library."""
        return lib.call(name, *args, variant=self.variant)

    # -- lifetime ------------------------------------------------------------
    def close(self):
        if getattr(self, "h", None):
            lib.load(self.variant).gfx_fluid_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001 -- interpreter shutdown
            pass

    # -- geometry ------------------------------------------------------------
    def geometry(self, axis):
        m = int(self.config.n_cells[axis]) + 2 * int(self.config.n_ghost_layers)
        c, wl, wr = (np.zeros(m) for _ in range(3))
        self.call("gfx_fluid_geometry", self.h, axis, c.ctypes.data_as(ctypes.c_void_p),
                 wl.ctypes.data_as(ctypes.c_void_p), wr.ctypes.data_as(ctypes.c_void_p))
        return c, wl, wr

    # -- Fluid_P_I ------------------------------------------------------------
    def compute_from_primitive(self, prim):
        """ComputeFromPrimitive on every value (after the periodic exchange);
        prim: [N, V1, V2, V3, E] over the ghost-inclusive brick."""
        torch = _torch()
        p = torch.as_tensor(np.ascontiguousarray(prim) if isinstance(prim, np.ndarray) else prim,
                            dtype=torch.float64, device=self.device).contiguous()
        assert tuple(p.shape) == (5,) + self.config.shape
        self.call("gfx_fluid_from_primitive", self.h, _ptr(p), _ptr(self.U), _stream())
        return self.U

    def set_conserved(self, U):
        """The state from conserved values: copied in, then ComputeFromConserved
        (floors, DS), so that the next step starts from these values."""
        torch = _torch()
        self.U.copy_(torch.as_tensor(U, dtype=torch.float64))
        self.call("gfx_fluid_to_primitive", self.h, _ptr(self.U), None, None, _stream())
        return self.U

    def compute_from_conserved(self, detect_features=False, primitive=False, aux=False):
        """ComputeFromConserved (floors U in place); optionally returns the
        primitives [5][...] and (P, CS, SB)."""
        torch = _torch()
        prim = torch.empty((5,) + self.config.shape, dtype=torch.float64,
                           device=self.device) if primitive else None
        ax = torch.empty((3,) + self.config.shape, dtype=torch.float64,
                         device=self.device) if aux else None
        self.call("gfx_fluid_to_primitive", self.h, _ptr(self.U), _ptr(prim), _ptr(ax), _stream())
        if detect_features:
            self.detect_features()
        return prim, ax

    def detect_features(self):
        self.call("gfx_fluid_detect_features", self.h, _ptr(self.U), _stream())

    def clear_features(self):
        self.call("gfx_fluid_clear_features", self.h, _stream())

    def features(self):
        """DIFFUSIVE_FLUX_I bits (bit d = direction d) over every value."""
        torch = _torch()
        f = torch.zeros(self.config.shape, dtype=torch.uint8, device=self.device)
        self.call("gfx_fluid_get_features", self.h, _ptr(f), _stream())
        return f

    def new_fluence(self):
        torch = _torch()
        return torch.zeros((6, 6, self.face_size), dtype=torch.float64, device=self.device)

    # -- increment, step, time step --------------------------------------------
    def increment(self, K, time_step, weight_rk=1.0, fluence=None):
        self.call("gfx_fluid_increment", self.h, _ptr(self.U), _ptr(K), float(time_step),
                 float(weight_rk), _ptr(fluence), _stream())
        return K

    def step(self, time_step, fluence=None):
        self.call("gfx_fluid_step", self.h, _ptr(self.U), float(time_step), _ptr(fluence),
                 _stream())

    def step_sources(self, time_step, fluence=None, sources=None):
        """The step of `step` (the same state bit for bit) with the reference's
        Sources records (Step_RK_C_ASC ApplyDivergence_C / RecordDivergenceKernel,
        ApplyGravity_F): a [10, *shape] tensor of the divergence sources of
        D, S_1, S_2, S_3, G, DS, then Gravitational_G and Gravitational_S_D 1-3."""
        torch = _torch()
        if sources is None:
            sources = torch.empty((N_SOURCES,) + tuple(self.config.shape), dtype=torch.float64,
                                  device=self.device)
        self.call("gfx_fluid_step_sources", self.h, _ptr(self.U), float(time_step),
                  _ptr(fluence), _ptr(sources), _stream())
        return sources

    def step_host(self, U_host, time_step, fluence_host=None):
        """One step on a host (ideally pinned) tensor: copy in, step, copy out."""
        self.call("gfx_fluid_step_host", self.h, _ptr(U_host), float(time_step),
                 _ptr(fluence_host))

    def step_timed(self, time_step, fluence=None):
        """One step with CUDA events around each launch; returns the device
        milliseconds of (features, stage 1, stage 2, ghost refresh)."""
        ms = (ctypes.c_double * 4)()
        self.call("gfx_fluid_step_timed", self.h, _ptr(self.U), float(time_step), _ptr(fluence),
                 ms, _stream())
        return tuple(ms)

    def set_tuning(self, z_chunk=0, adjoint_segment=0, tile_rows=0):
        """Speed knobs that leave results unchanged (genasis_b200.autotune):
        pencil length, adjoint sweep segment, tile rows (8 or 16)."""
        self.call("gfx_fluid_set_tuning", self.h, int(z_chunk), int(adjoint_segment),
                 int(tile_rows))
        self.tuning = (int(z_chunk), int(adjoint_segment), int(tile_rows))

    def totals(self, U=None):
        """sum U dV over the proper cells for the six conserved fields
        (the conservation tallies), as a numpy array."""
        out = np.zeros(6)
        self.call("gfx_fluid_totals", self.h, _ptr(self.U if U is None else U),
                 out.ctypes.data_as(ctypes.c_void_p), _stream())
        return out

    def check_state(self, U=None):
        """Raises GfxError (GFX_ERR_STATE) if a proper cell of U (default: the
        box's state) holds a non-finite value."""
        self.call("gfx_fluid_check_state", self.h, _ptr(self.U if U is None else U), _stream())

    def kernel_launches(self):
        n = ctypes.c_longlong()
        self.call("gfx_fluid_kernel_launches", self.h, ctypes.byref(n))
        return int(n.value)

    def compute_time_step(self, i_cycle=0):
        dt = ctypes.c_double()
        self.call("gfx_fluid_timestep", self.h, _ptr(self.U), int(i_cycle), ctypes.byref(dt),
                 _stream())
        return dt.value

    def evolve(self, finish_time, time=0.0, i_cycle=0, max_cycles=2**31 - 1):
        t = ctypes.c_double()
        c = ctypes.c_int()
        self.call("gfx_fluid_evolve", self.h, _ptr(self.U), float(time), int(i_cycle),
                 float(finish_time), int(max_cycles), ctypes.byref(t), ctypes.byref(c),
                 _stream())
        return t.value, c.value

    def evolve_timed(self, finish_time, time=0.0, i_cycle=0, max_cycles=2**31 - 1):
        """evolve, and the device milliseconds of its work (CUDA events the
        library records just before its first and after its last launch):
        returns (time, cycle, ms)."""
        t = ctypes.c_double()
        c = ctypes.c_int()
        ms = ctypes.c_double()
        self.call("gfx_fluid_evolve_timed", self.h, _ptr(self.U), float(time), int(i_cycle),
                  float(finish_time), int(max_cycles), ctypes.byref(t), ctypes.byref(c),
                  ctypes.byref(ms), _stream())
        return t.value, c.value, ms.value


class Step_RK2_C_ASC:
    """Step_RK_C_ASC_Template % Compute (Step_RK_C_ASC__Template.f90:504-542)
    on a FluidBox's current."""

    def __init__(self, box: FluidBox, record_sources=False):
        self.box = box
        self.boundary_fluence = box.new_fluence()
        # the current's Sources (Sources_F) when the step records them
        self.sources = None
        if record_sources:
            torch = _torch()
            self.sources = torch.zeros((N_SOURCES,) + tuple(box.config.shape),
                                       dtype=torch.float64, device=box.device)

    def compute(self, time, time_step):
        del time  # the RK2 stages of this fluid do not depend on the time
        if self.sources is not None:
            self.box.step_sources(time_step, self.boundary_fluence, self.sources)
        else:
            self.box.step(time_step, self.boundary_fluence)


class IncrementDivergence_FV:
    """IncrementDivergence_FV_Form % Compute (IncrementDivergence_FV__Form.f90:344-412)."""

    def __init__(self, box: FluidBox):
        self.box = box
        self.boundary_fluence = box.new_fluence()

    def compute(self, increment, time_step, weight_rk):
        """increment: [6][...] device tensor, assumed cleared by the caller as
        the reference assumes."""
        return self.box.increment(increment, time_step, weight_rk, self.boundary_fluence)


class Integrator_C_PS:
    """The integrator's ComputeTimeStep and Evolve loop (Integrator_Template.f90)."""

    def __init__(self, box: FluidBox, finish_time, finish_cycle=2**31 - 1):
        self.box = box
        self.time = 0.0
        self.i_cycle = 0
        self.finish_time = finish_time
        self.finish_cycle = finish_cycle

    def compute_time_step(self):
        return self.box.compute_time_step(self.i_cycle)

    def evolve(self):
        self.time, self.i_cycle = self.box.evolve(
            self.finish_time, self.time, self.i_cycle, self.finish_cycle - self.i_cycle)
        return self.time, self.i_cycle
