"""Verification case setups (same API as CFD-demo's src/cfd_demo/cases.py)."""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .boundary import FixedState, SlipWall
from .mesh import rectangle_mesh
from .solver import DEFAULT_CFL, EulerSolver, SolverConfig

# Two-dimensional Sod shock tube (cases.py:15-22)
SOD_GAMMA = 1.4
SOD_LEFT = (1.0, 0.0, 0.0, 1.0)  # (rho, u, v, p) for x < 0.5
SOD_RIGHT = (0.125, 0.0, 0.0, 0.1)  # (rho, u, v, p) for x > 0.5
SOD_DISCONTINUITY = 0.5
SOD_X_RANGE = (0.0, 1.0)
SOD_Y_RANGE = (0.0, 0.1)
SOD_FINAL_TIME = 0.2


@dataclass(frozen=True, eq=False)
class SodShockTube:
    solver: EulerSolver
    initial_state: np.ndarray
    final_time: float


def sod_boundaries(left=SOD_LEFT, right=SOD_RIGHT, gamma: float = SOD_GAMMA) -> dict:
    return {"left": FixedState.from_primitive(*left, gamma=gamma), "right": FixedState.from_primitive(*right, gamma=gamma),
            "bottom": SlipWall(), "top": SlipWall()}


def sod_shock_tube(nx: int = 200, ny: int = 20, *, flux: str, limiter: str, cfl: float = DEFAULT_CFL,
                   precision: str = "fp64", **solver_options) -> SodShockTube:
    """The Sod shock tube on nx*ny rectangles split into triangles, slip walls
    at top and bottom, the initial states as fixed exterior states at the ends
    (cases.py:31-44). ``precision`` selects the plain FP64 or the FP32-mixed form."""
    mesh = rectangle_mesh(nx, ny, SOD_X_RANGE, SOD_Y_RANGE)
    bcs = sod_boundaries()
    config = SolverConfig(flux=flux, limiter=limiter, gamma=SOD_GAMMA, cfl=cfl, precision=precision)
    solver = EulerSolver(mesh, bcs, config, **solver_options)
    on_left = solver.geometry.centroid[:, 0] < SOD_DISCONTINUITY
    element_state = np.where(on_left[:, None], np.array(bcs["left"].state), np.array(bcs["right"].state))
    initial_state = np.broadcast_to(element_state[None], solver.state_shape).copy()
    return SodShockTube(solver=solver, initial_state=initial_state, final_time=SOD_FINAL_TIME)
