"""Many independent bricks advanced together (C ABI gfx_fluid_batch_*).

Each brick is a FluidBox (its own Fluid_P_I current and CFL time step); the
batch advances all of them with one persistent launch per RK stage, the
cycle replayed from one CUDA graph.  The reference runs such bricks one
program (or rank) each, every cycle being Integrator % Evolve's ComputeCycle
(Integrator_Template.f90:291-346)."""
import ctypes

import numpy as np

from . import lib
from .fluid import FluidBox, _stream


class FluidBatch:
    def __init__(self, configs, device=None, variant=None):
        self.variant = variant or lib.default_variant()
        self.boxes = [FluidBox(c, device=device, variant=self.variant) for c in configs]
        self.h = None

    def _call(self, name, *args):
        return lib.call(name, *args, variant=self.variant)

    def set_pencil_length(self, z_chunk, tile_rows=None):
        """The z length of the cell pencils of every brick's work items (0 =
        32 planes) and, if given, the tile rows (8 or 16); rebuilds the
        batch's work list on its next use."""
        for b in self.boxes:
            _, seg, rows = getattr(b, "tuning", (0, 0, 0))
            b.set_tuning(z_chunk, seg, rows if tile_rows is None else tile_rows)
        if self.h is not None:
            lib.load(self.variant).gfx_fluid_batch_destroy(self.h)
            self.h = None

    def set_primitives(self, prims):
        for box, prim in zip(self.boxes, prims):
            box.compute_from_primitive(prim)

    def _ensure(self):
        if self.h is not None:
            return
        n = len(self.boxes)
        hs = (ctypes.c_void_p * n)(*[b.h.value for b in self.boxes])
        us = (ctypes.c_void_p * n)(*[b.U.data_ptr() for b in self.boxes])
        h = ctypes.c_void_p()
        self._call("gfx_fluid_batch_create", n, hs, us, ctypes.byref(h))
        self.h = h

    def set_clocks(self, time=0.0, i_cycle=0):
        self._ensure()
        self._call("gfx_fluid_batch_set_clocks", self.h, float(time), int(i_cycle))

    def evolve(self, finish_time=1e300, n_cycles=1):
        """Advances every brick by its own CFL steps until finish_time or
        n_cycles more cycles (asynchronous on the current stream)."""
        self._ensure()
        self._call("gfx_fluid_batch_evolve", self.h, float(finish_time), int(n_cycles), _stream())

    def clocks(self):
        self._ensure()
        n = len(self.boxes)
        t = np.zeros(n)
        c = np.zeros(n, dtype=np.int32)
        self._call("gfx_fluid_batch_clocks", self.h, t.ctypes.data_as(ctypes.c_void_p),
                 c.ctypes.data_as(ctypes.c_void_p), _stream())
        return t, c

    def kernel_launches(self):
        self._ensure()
        n = ctypes.c_longlong()
        self._call("gfx_fluid_batch_kernel_launches", self.h, ctypes.byref(n))
        return int(n.value)

    def close(self):
        if self.h is not None:
            lib.load(self.variant).gfx_fluid_batch_destroy(self.h)
            self.h = None
        for b in self.boxes:
            b.close()

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001 -- interpreter shutdown
            pass


def shard_bricks(configs, world, rank):
    """The bricks that rank `rank` of `world` advances when a set of
    independent bricks is split over GPUs, one rank per GPU, as the
    reference gives each brick to its own program or rank.  The bricks are
    taken in decreasing order of proper cells (ties by index), and each goes
    to the rank with the fewest cells so far (ties to the lower rank).  Every
    rank computes the same split from the same list, so the split needs no
    collective.  The indices come back in increasing order."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank %r of a world of %r" % (rank, world))
    cells = [int(c.n_proper) for c in configs]
    load = [0] * world
    owner = [0] * len(cells)
    for i in sorted(range(len(cells)), key=lambda j: (-cells[j], j)):
        r = min(range(world), key=lambda q: (load[q], q))
        owner[i] = r
        load[r] += cells[i]
    return [i for i in range(len(cells)) if owner[i] == rank]
