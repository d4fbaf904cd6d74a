"""genasis_b200 -- B200-native finite-volume step for the GenASiS ideal-gas
fluid (Fluid_P_I): hand-written sm_100a kernels behind the reference's
Step_RK / IncrementDivergence_FV call surface (C ABI: include/gfx_fluid.h)."""
from .config import FluidConfig  # noqa: F401
from .lib import GfxError  # noqa: F401

__all__ = ["FluidConfig", "GfxError", "FluidBox", "Step_RK2_C_ASC", "IncrementDivergence_FV",
           "Integrator_C_PS"]


def __getattr__(name):
    if name in ("FluidBox", "Step_RK2_C_ASC", "IncrementDivergence_FV", "Integrator_C_PS"):
        from . import fluid

        return getattr(fluid, name)
    raise AttributeError(name)
