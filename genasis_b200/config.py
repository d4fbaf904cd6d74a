"""FluidConfig: the parameters of one single-brick Fluid_P_I box.

Field names follow the reference's GetParameter names (nCells -> n_cells,
MinCoordinate -> min_coordinate, RiemannSolverType -> riemann_solver, ...);
defaults are the reference defaults:
  ChartHeader_SL__Form.f90:345-366 (nGhostLayers 2), Chart_Template.f90:178-192
  ([0,1] per axis), Fluid_ASC__Form.f90:128-177 (HLLC, PRIMITIVE, limiter 1.4),
  Fluid_P_I__Form.f90:210 (gamma 1.4), IncrementDivergence_FV__Form.f90:239
  (ReconstructionType LINEAR), FluidFeatures_ASC__Form.f90:61-65
  (ShockThreshold 0.1), Integrator_C_PS__Form.f90:136 (Courant 0.7),
  IntegratorHeader_Form.f90:95 (nRampCycles 100).
"""
import ctypes
from dataclasses import dataclass, field

BC = {"OUTFLOW": 0, "REFLECTING": 1, "PERIODIC": 2}
RIEMANN = {"HLL": 0, "HLLC": 1}
RECONSTRUCTION = {"LINEAR": 0, "PARABOLIC": 1}


class GfxConfig(ctypes.Structure):
    """Mirror of gfx_fluid_config in include/gfx_fluid.h."""
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


@dataclass
class FluidConfig:
    n_cells: tuple = (32, 32, 32)
    n_ghost_layers: int = 2
    min_coordinate: tuple = (0.0, 0.0, 0.0)
    max_coordinate: tuple = (1.0, 1.0, 1.0)
    # [axis][inner, outer]
    boundary: tuple = (("OUTFLOW", "OUTFLOW"),) * 3
    riemann_solver: str = "HLLC"
    use_limiter: bool = True
    limiter_parameter: float = 1.4
    adiabatic_index: float = 1.4
    shock_threshold: float = 0.1
    courant_factor: float = 0.7
    baryon_density_min: float = 0.0
    uniform_acceleration: float = 0.0
    n_ramp_cycles: int = 100
    reconstruction: str = "LINEAR"  # ReconstructionType: LINEAR or PARABOLIC

    @property
    def shape(self):
        """Ghost-inclusive (z, y, x) shape of one field."""
        g = self.n_ghost_layers
        return tuple(int(self.n_cells[2 - d]) + 2 * g for d in range(3))

    @property
    def proper(self):
        """Index of the proper cells in a ghost-inclusive field."""
        g = self.n_ghost_layers
        return tuple(slice(g, g + int(self.n_cells[2 - d])) for d in range(3))

    @property
    def n_proper(self):
        return int(self.n_cells[0]) * int(self.n_cells[1]) * int(self.n_cells[2])

    def to_c(self):
        c = GfxConfig()
        for d in range(3):
            c.n_cells[d] = int(self.n_cells[d])
            c.min_coordinate[d] = float(self.min_coordinate[d])
            c.max_coordinate[d] = float(self.max_coordinate[d])
            for s in range(2):
                b = self.boundary[d][s]
                c.boundary[d][s] = BC[b] if isinstance(b, str) else int(b)
        c.n_ghost_layers = int(self.n_ghost_layers)
        rs = self.riemann_solver
        c.riemann_solver = RIEMANN[rs] if isinstance(rs, str) else int(rs)
        c.use_limiter = int(bool(self.use_limiter))
        c.limiter_parameter = float(self.limiter_parameter)
        c.adiabatic_index = float(self.adiabatic_index)
        c.shock_threshold = float(self.shock_threshold)
        c.courant_factor = float(self.courant_factor)
        c.baryon_density_min = float(self.baryon_density_min)
        c.uniform_acceleration = float(self.uniform_acceleration)
        c.n_ramp_cycles = int(self.n_ramp_cycles)
        rc = self.reconstruction
        c.reconstruction = RECONSTRUCTION[rc] if isinstance(rc, str) else int(rc)
        return c
