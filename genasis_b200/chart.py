"""A chart of several bricks on one device (C ABI gfx_fluid_chart_*).

The reference's distributed single-level chart, Chart_SLD (Chart_SLD__Form.f90),
splits one domain into nBricks equal bricks (nCellsBrick = nCells / nBricks,
Chart_Template.f90:440-460), one per MPI rank, and exchanges the bricks'
ghost layers every stage.  FluidChart keeps every brick's state in device
memory of its own ([6][nV] of the brick, ghosts included, brick b = ix + nx
(iy + ny iz)) and steps all bricks together: one launch per stage over the
whole chart, a halo cell across a brick face read from the neighbouring
brick.  Its results on every cell are those of one brick of the whole chart,
bit for bit; `gather` assembles the chart's proper cells for comparison.
"""
import ctypes

import numpy as np

from . import lib
from .config import FluidConfig
from .fluid import _ptr, _stream, _torch


class FluidChart:
    def __init__(self, config: FluidConfig, n_bricks=(2, 2, 2), device=None, variant=None):
        torch = _torch()
        if not torch.cuda.is_available():
            raise RuntimeError("FluidChart needs a CUDA device (there is no CPU path)")
        self.config = config
        self.n_bricks = tuple(int(b) for b in n_bricks)
        self.variant = variant or lib.default_variant()
        self.device = torch.device(device) if device is not None else torch.device("cuda")
        self._c = config.to_c()
        nb = (ctypes.c_int * 3)(*self.n_bricks)
        h = ctypes.c_void_p()
        self.call("gfx_fluid_chart_create", ctypes.byref(self._c), nb, ctypes.byref(h))
        self.h = h
        n = ctypes.c_int()
        self.call("gfx_fluid_chart_n_bricks", self.h, ctypes.byref(n))
        self.brick_cells = tuple(int(config.n_cells[a]) // self.n_bricks[a] for a in range(3))
        g = int(config.n_ghost_layers)
        shape = tuple(self.brick_cells[2 - d] + 2 * g for d in range(3))
        self.U = [torch.zeros((6,) + shape, dtype=torch.float64, device=self.device)
                  for _ in range(n.value)]
        self.index = []
        for b in range(n.value):
            ib = (ctypes.c_int * 3)()
            self.call("gfx_fluid_chart_brick", self.h, b, None, ib)
            self.index.append(tuple(ib))
        arr = (ctypes.c_void_p * len(self.U))(*[u.data_ptr() for u in self.U])
        self.call("gfx_fluid_chart_bind", self.h, arr)

    def call(self, name, *args):
        return lib.call(name, *args, variant=self.variant)

    def close(self):
        if getattr(self, "h", None):
            lib.load(self.variant).gfx_fluid_chart_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001 -- interpreter shutdown
            pass

    # -- brick <-> chart layouts -------------------------------------------------
    def _region(self, b):
        """Slices (z, y, x) of brick b's ghost-inclusive block in the chart's
        ghost-inclusive layout."""
        g = int(self.config.n_ghost_layers)
        out = []
        for d in (2, 1, 0):
            o = self.index[b][d] * self.brick_cells[d]
            out.append(slice(o, o + self.brick_cells[d] + 2 * g))
        return tuple(out)

    def _proper_region(self, b):
        g = int(self.config.n_ghost_layers)
        out = []
        for d in (2, 1, 0):
            o = self.index[b][d] * self.brick_cells[d] + g
            out.append(slice(o, o + self.brick_cells[d]))
        return tuple(out)

    def from_primitive(self, prim):
        """ComputeFromPrimitive of every brick from the chart's primitive
        array prim ([5] + the chart's ghost-inclusive shape): brick b gets its
        block of it, ghosts included."""
        torch = _torch()
        p = np.ascontiguousarray(prim)
        bricks = [torch.as_tensor(np.ascontiguousarray(p[(slice(None),) + self._region(b)]),
                                  dtype=torch.float64, device=self.device)
                  for b in range(len(self.U))]
        arr = (ctypes.c_void_p * len(bricks))(*[t.data_ptr() for t in bricks])
        self.call("gfx_fluid_chart_from_primitive", self.h, arr, _stream())
        torch.cuda.current_stream().synchronize()

    def set_conserved(self, U):
        """The chart's state from conserved values U ([6] + the chart's
        ghost-inclusive shape), then ComputeFromConserved and the features."""
        torch = _torch()
        for b, u in enumerate(self.U):
            u.copy_(torch.as_tensor(np.ascontiguousarray(np.asarray(U)[(slice(None),) +
                                                                     self._region(b)])))
        self.call("gfx_fluid_chart_set_conserved", self.h, _stream())

    def gather(self, ghosts=False):
        """The chart's state ([6] + the chart's ghost-inclusive shape)
        assembled from the bricks' proper cells; the chart's ghosts are left
        zero, or (ghosts) taken from the bricks along the chart's faces."""
        g = int(self.config.n_ghost_layers)
        out = np.zeros((6,) + self.config.shape)
        hosts = [u.cpu().numpy() for u in self.U]
        if ghosts:
            for b, host in enumerate(hosts):
                out[(slice(None),) + self._region(b)] = host
        inner = tuple(slice(g, g + self.brick_cells[d]) for d in (2, 1, 0))
        for b, host in enumerate(hosts):
            out[(slice(None),) + self._proper_region(b)] = host[(slice(None),) + inner]
        return out

    # -- time step, step, evolve ---------------------------------------------------
    def compute_time_step(self, i_cycle=0):
        dt = ctypes.c_double()
        self.call("gfx_fluid_chart_timestep", self.h, int(i_cycle), ctypes.byref(dt), _stream())
        return dt.value

    def new_fluence(self):
        torch = _torch()
        out = []
        for _ in self.U:
            n = self.brick_cells
            fs = max(n[1] * n[2], n[0] * n[2], n[0] * n[1])
            out.append(torch.zeros((6, 6, fs), dtype=torch.float64, device=self.device))
        return out

    def step(self, time_step, fluence=None):
        arr = None
        if fluence is not None:
            arr = (ctypes.c_void_p * len(fluence))(*[f.data_ptr() for f in fluence])
        self.call("gfx_fluid_chart_step", self.h, float(time_step), arr, _stream())

    def evolve(self, finish_time, time=0.0, i_cycle=0, max_cycles=2**31 - 1):
        t = ctypes.c_double()
        c = ctypes.c_int()
        self.call("gfx_fluid_chart_evolve", self.h, float(time), int(i_cycle),
                  float(finish_time), int(max_cycles), ctypes.byref(t), ctypes.byref(c),
                  _stream())
        return t.value, c.value

    def kernel_launches(self):
        n = ctypes.c_longlong()
        self.call("gfx_fluid_chart_kernel_launches", self.h, ctypes.byref(n))
        return int(n.value)

    def totals(self):
        """sum U dV of the six conserved fields over the chart's proper cells."""
        out = np.zeros(6)
        for b, u in enumerate(self.U):
            h = ctypes.c_void_p()
            self.call("gfx_fluid_chart_brick", self.h, b, ctypes.byref(h), None)
            t = np.zeros(6)
            self.call("gfx_fluid_totals", h, _ptr(u), t.ctypes.data_as(ctypes.c_void_p),
                      _stream())
            out += t
        return out
