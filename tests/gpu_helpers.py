"""Shared helpers of the GPU tests: run the CUDA path (through the C ABI)
and the CPU oracle on the same inputs and compare."""
import numpy as np

from oracle.oracle import Oracle

# The parity bar: per step, per conserved field,
# max |U_gpu - U_oracle| / max |U_oracle| <= 1e-12 over proper cells.
PARITY_RTOL = 1e-12


def to_np(t):
    return t.detach().cpu().numpy()


def field_errors(a, b, index):
    """Max abs difference per field over `index`, relative to the field's max."""
    out = []
    for f in range(a.shape[0]):
        x, y = a[f][index], b[f][index]
        scale = max(float(np.abs(y).max()), 1e-300)
        out.append(float(np.abs(x - y).max()) / scale)
    return out


def assert_parity(gpu, ref, cfg, what="", rtol=PARITY_RTOL, index=None):
    idx = cfg.proper if index is None else index
    errs = field_errors(gpu, ref, idx)
    assert max(errs) <= rtol, "%s: relative errors per field %s" % (what, errs)
    return errs


def make_pair(cfg, prim):
    from genasis_b200.fluid import FluidBox

    box = FluidBox(cfg)
    o = Oracle(cfg)
    box.compute_from_primitive(prim)
    o.set_primitive(prim)
    return box, o
