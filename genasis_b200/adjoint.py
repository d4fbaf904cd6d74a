"""Discrete adjoint of the RK2 step, and a torch.autograd.Function over it.

gfx_fluid_step_adjoint (include/gfx_fluid.h) is the hand-written reverse of
one step with dt held fixed; this module chains it over a run with per-step
checkpointing (the state before every step is kept; the adjoint recomputes
the stages of a step from its checkpoint) and exposes the run to
torch.autograd for gradient checks:

    U_final = Evolve.apply(U0, box, dts, detect_first)
    J = objective(U_final); J.backward()   # U0.grad = dJ / dU0

The reference has no adjoint; the forward it differentiates is
Step_RK_C_ASC_Template % Compute (Step_RK_C_ASC__Template.f90:504-542).
"""
from . import lib
from .fluid import FluidBox, _ptr, _stream, _torch


def step_adjoint(box: FluidBox, U_n, dt, lam_np1, lam_n=None, U_np1=None,
                 detect_features=True):
    """lam_n = (dU_np1 / dU_n)^T lam_np1 for one step of size dt from U_n.

    U_n, lam_np1, U_np1 (optional: recomputed when None) and lam_n are
    [6][...] float64 device tensors of the brick's ghost-inclusive shape."""
    torch = _torch()
    if lam_n is None:
        lam_n = torch.empty_like(lam_np1)
    box.call("gfx_fluid_step_adjoint", box.h, _ptr(U_n.contiguous()), float(dt),
             _ptr(lam_np1.contiguous()), _ptr(lam_n), _ptr(U_np1), int(bool(detect_features)),
             _stream())
    return lam_n


BRANCH_KINDS = ("slope_zero", "slope_left", "slope_right", "slope_centred", "ap_0", "ap_left",
                "ap_right", "am_0", "am_left", "am_right", "hllc_centre", "ac_nonnegative",
                "md_positive", "floored", "flags")


def step_branches(box: FluidBox, U_n, dt, detect_features=True):
    """The branch signature of one forward step from U_n
    (gfx_fluid_step_branches): (hash, decisions, counts per kind)."""
    import ctypes

    import numpy as np

    out = np.zeros(2 + len(BRANCH_KINDS), dtype=np.uint64)
    box.call("gfx_fluid_step_branches", box.h, _ptr(U_n.contiguous()), float(dt),
             int(bool(detect_features)), out.ctypes.data_as(ctypes.c_void_p), _stream())
    return int(out[0]), int(out[1]), out[2:].astype(np.int64)


def branch_signature(box: FluidBox, U0, dts, detect_first=False):
    """The branches of the run of steps dts from U0 (the forward of
    run_forward): the hash of every step's decisions (summed modulo 2^64)
    and the counts per kind, summed over the steps."""
    import numpy as np

    prepare_state(box, U0, detect_first)
    h, counts = 0, np.zeros(len(BRANCH_KINDS), dtype=np.int64)
    for i, dt in enumerate(dts):
        hi, _, ci = step_branches(box, box.U, dt, detect_first or i > 0)
        h = (h + hi) % (1 << 64)
        counts += ci
        box.step(float(dt))
    return h, counts


def prepare_state(box: FluidBox, U0, detect_first):
    """Loads U0 as the box's state from conserved values, with the shock
    features of U0 (detect_first) or zero features (the first step after
    initialisation from primitives)."""
    box.U.copy_(U0)
    box.call("gfx_fluid_to_primitive", box.h, _ptr(box.U), None, None, _stream())
    if detect_first:
        box.detect_features()
    else:
        box.clear_features()


def run_forward(box: FluidBox, U0, dts, detect_first=False, keep=True):
    """The steps of sizes dts from U0; returns the final state and, if keep,
    the checkpoints [U^0, ..., U^n] (device tensors)."""
    prepare_state(box, U0, detect_first)
    checkpoints = [box.U.clone()] if keep else None
    for dt in dts:
        box.step(float(dt))
        if keep:
            checkpoints.append(box.U.clone())
    return box.U.clone(), checkpoints


def run_adjoint(box: FluidBox, checkpoints, dts, lam_final, detect_first=False):
    """lam^0 from lam^n through the stored checkpoints, last step first."""
    torch = _torch()
    lam = lam_final.contiguous().clone()
    other = torch.empty_like(lam)
    for k in range(len(dts) - 1, -1, -1):
        step_adjoint(box, checkpoints[k], dts[k], lam, other, checkpoints[k + 1],
                     detect_features=(k > 0 or detect_first))
        lam, other = other, lam
    return lam


def _evolve_function():
    torch = _torch()

    class Evolve(torch.autograd.Function):
        """U0 -> U^n over the steps dts on the box, differentiable in U0 by
        the hand-written adjoint (per-step checkpoints, stage recomputation)."""

        @staticmethod
        def forward(ctx, U0, box, dts, detect_first=False):
            out, checkpoints = run_forward(box, U0.detach().contiguous(), dts, detect_first)
            ctx.box = box
            ctx.dts = list(dts)
            ctx.detect_first = detect_first
            ctx.checkpoints = checkpoints
            return out

        @staticmethod
        def backward(ctx, lam):
            g = run_adjoint(ctx.box, ctx.checkpoints, ctx.dts, lam, ctx.detect_first)
            ctx.checkpoints = None
            return g, None, None, None

    return Evolve


_EVOLVE = None


def __getattr__(name):
    global _EVOLVE
    if name == "Evolve":
        if _EVOLVE is None:
            _EVOLVE = _evolve_function()
        return _EVOLVE
    raise AttributeError(name)


def cell_volumes(box: FluidBox):
    """dV of every value of the brick (ghost-inclusive shape), from the
    chart's widths."""
    torch = _torch()
    w = []
    for axis in range(3):
        _, wl, wr = box.geometry(axis)
        w.append(torch.as_tensor(wl + wr, dtype=torch.float64, device=box.device))
    return w[2][:, None, None] * w[1][None, :, None] * w[0][None, None, :]


def density_squared(box: FluidBox, U):
    """J = sum over proper cells of rho^2 dV (the adjoint benchmark's objective)."""
    dv = cell_volumes(box)
    p = box.config.proper
    return (U[0][p] ** 2 * dv[p]).sum()

