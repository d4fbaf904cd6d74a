"""Writes the regression fixtures of tests/golden/ from the oracle.

Each fixture holds a small seeded problem (its configuration, initial
primitives and the CFL time steps of its run), the conserved state after the
run, the last step's boundary fluence and the final feature flags.  The
reference cannot be run here, so these pin the oracle (and, through the GPU
tests, the CUDA path) against this recorded output: a change of either shows
up as a difference.

    python tests/golden/make_golden.py
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from genasis_b200 import problems  # noqa: E402
from genasis_b200.config import FluidConfig  # noqa: E402
from oracle.oracle import Oracle  # noqa: E402


def cases():
    sod_cfg = FluidConfig(n_cells=(12, 6, 6), riemann_solver="HLL", courant_factor=0.8,
                          n_ramp_cycles=1)
    sod = problems.riemann(sod_cfg, 1.0, 1.0, (0, 0, 0), 0.125, 0.1, (0, 0, 0), (0.5, 0, 0),
                           (1.0, 0, 0))
    sine_cfg, sine = problems.sine_wave(8, riemann_solver="HLLC")
    rt_cfg, rt = problems.rayleigh_taylor(shape=(8, 8, 12), seed=3)
    mix = FluidConfig(n_cells=(10, 7, 9), riemann_solver="HLLC", courant_factor=0.8,
                      n_ramp_cycles=1,
                      boundary=(("OUTFLOW", "REFLECTING"), ("PERIODIC", "PERIODIC"),
                                ("REFLECTING", "OUTFLOW")))
    return {
        "sod_hll_12x6x6": (sod_cfg, sod, 3),
        "sine_hllc_8": (sine_cfg, sine, 2),
        "rt_hllc_gravity_8x8x12": (rt_cfg, rt, 2),
        "random_hllc_mixed_10x7x9": (mix, problems.random_state(mix, seed=21), 3),
    }


def run(cfg, prim, n_steps):
    o = Oracle(cfg)
    o.set_primitive(prim)
    dts = []
    fluence = o.new_fluence()
    for i in range(n_steps):
        dts.append(o.timestep(i))
        fluence[:] = 0.0
        o.step(dts[-1], fluence)
    return o, np.array(dts), fluence


def config_dict(cfg):
    return {k: getattr(cfg, k) for k in cfg.__dataclass_fields__}


def main():
    for name, (cfg, prim, n) in cases().items():
        o, dts, fluence = run(cfg, prim, n)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), prim=prim, dts=dts,
                            U=o.conserved(), fluence=fluence, features=o.features(),
                            config=json.dumps(config_dict(cfg)))
        print(name, n, "steps", dts)


if __name__ == "__main__":
    main()
