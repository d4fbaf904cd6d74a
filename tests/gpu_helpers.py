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


def quantity_errors(a, b, index):
    """Max abs difference per field over `index`, relative to the size of the
    quantity it belongs to: D, G and DS to their own field's max, each
    momentum component to the largest of the three (the momentum vector's
    scale).  The bar of the speed build, whose rounding differs from the
    reference's: a momentum component that carries only round-off-sized
    values (a transverse component of a planar flow) has no scale of its own."""
    scale = [max(float(np.abs(b[f][index]).max()), 1e-300) for f in range(b.shape[0])]
    s = max(scale[1:4])
    scale[1:4] = [s, s, s]
    return [float(np.abs(a[f][index] - b[f][index]).max()) / scale[f]
            for f in range(a.shape[0])]


def make_pair(cfg, prim, variant=None):
    from genasis_b200.fluid import FluidBox

    box = FluidBox(cfg, variant=variant)
    o = Oracle(cfg)
    box.compute_from_primitive(prim)
    o.set_primitive(prim)
    return box, o
