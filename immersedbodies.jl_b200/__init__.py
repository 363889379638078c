"""immersedbodies.jl_b200 -- ImmersedBodies.jl's IBPM time step on one B200.

The CUDA library (csrc/, built into lib/libibpm_b200.so) holds the time step;
this package mirrors the reference's problem/solver API on the host
(src/problem.jl, src/curves.jl, src/solver.jl, src/io/io.jl) and drives the
library through its C ABI (include/ibpm_b200.h).
"""
from . import curves as Curves
from . import configs
from . import warmstart
from .io import load_state, load_state_, save_state
from .problem import (CNAB, Bodies, CartesianGrid, Fluid, GridIndices, GridVelocity, MovingGrid, MovingRigidBody,
                      MultiDomainGrid, Panels, PanelState, Problem, RigidBodyTransform, State, StaticBody,
                      StaticGrid, boundary_force, boundary_total_force, default_gridstep, default_scheme, fluid_grid,
                      inc_time_index_, n_panels, set_time_index_, timestep, update_vars_, vorticity, x_velocity,
                      y_velocity)
from .solver import AbstractSolver, GpuCnabSolver, advance_, create_solver, getstate, solve, solve_
from .warmstart import WarmStartNet
from . import ensemble
from .ensemble import Ensemble

__all__ = [n for n in dir() if not n.startswith("_")]
