"""B200-native drop-in for the hot path of CFD-demo: the degree-4 nodal DG
right-hand side, limiters and SSP-RK3 step for the 2D Euler equations, as
hand-written sm_100a CUDA kernels behind a C ABI (include/cfd_b200.h),
driven from Python with PyTorch tensors as device buffers.

Same public names as ``cfd_demo``; ``SolverConfig`` adds ``precision``
("fp64" plain form, "fp32_mixed").
"""

from .boundary import ExactState, FixedState, SlipWall
from .cases import ObliqueShockCase, SodShockTube, oblique_shock, sod_shock_tube
from .fluxes import INTERFACE_FLUXES, get_interface_flux
from .limiters import LIMITER_FUNCTIONS, get_limiter_function
from .mesh import TriangleMesh, jittered_rectangle_mesh, rectangle_mesh, sheared_rectangle_mesh
from .solver import EulerSolver, RunResult, SolverConfig, SolverError, StepReport

__all__ = [
    "INTERFACE_FLUXES",
    "LIMITER_FUNCTIONS",
    "ObliqueShockCase",
    "EulerSolver",
    "ExactState",
    "FixedState",
    "RunResult",
    "SlipWall",
    "SodShockTube",
    "SolverConfig",
    "SolverError",
    "StepReport",
    "TriangleMesh",
    "get_interface_flux",
    "get_limiter_function",
    "jittered_rectangle_mesh",
    "oblique_shock",
    "rectangle_mesh",
    "sheared_rectangle_mesh",
    "sod_shock_tube",
]
