"""Checkpoint and restart of a brick's state (the reference's restart files,
Integrator_Template.f90:476-502 and 658-764, written through its Silo
GridImageStream there; here one compressed numpy archive per brick).

A checkpoint holds the configuration, the integrator's time and cycle and
the conserved state with its ghost values; a restart loads it into a new
FluidBox and continues as the uninterrupted run would (gfx_fluid_resume:
the next step detects the shock features of the loaded state), bit for bit.
"""
import json

import numpy as np

from . import lib
from .config import FluidConfig
from .fluid import FluidBox, _ptr, _torch

FORMAT = "gfx-fluid-checkpoint-1"


def save(box: FluidBox, path, time, i_cycle):
    """Writes box's state, time and cycle to path (.npz)."""
    cfg = {k: getattr(box.config, k) for k in box.config.__dataclass_fields__}
    np.savez_compressed(path, format=FORMAT, config=json.dumps(cfg), time=float(time),
                        i_cycle=int(i_cycle), U=box.U.detach().cpu().numpy())


def load(path, device=None):
    """Reads a checkpoint; returns (FluidBox with the state, time, cycle)."""
    z = np.load(path)
    if str(z["format"]) != FORMAT:
        raise ValueError("%s is not a %s file" % (path, FORMAT))
    cfg = FluidConfig(**json.loads(str(z["config"])))
    box = FluidBox(cfg, device=device)
    torch = _torch()
    box.U.copy_(torch.as_tensor(z["U"], dtype=torch.float64))
    box.call("gfx_fluid_resume", box.h, _ptr(box.U))
    return box, float(z["time"]), int(z["i_cycle"])
