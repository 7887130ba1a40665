"""Verification case setups (same API as CFD-demo's src/cfd_demo/cases.py),
plus the oblique-shock case that CFD-demo proposes in ADR 0011 / 0012 but
does not implement."""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .boundary import ExactState, FixedState, SlipWall
from .mesh import rectangle_mesh, sheared_rectangle_mesh
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


# Steady oblique shock over a compression corner (CFD-demo's proposed
# docs/adr/0011-oblique-shock-verification.md): dimensionless, gamma = 1.4,
# baseline (M1, theta) = (2, 10 deg). Domain 0 <= x <= length,
# x tan(theta) <= y <= x tan(theta) + height (sheared rectangle, ADR 0012).
# With length 1 and height 0.5 the baseline shock (beta = 39.3 deg) leaves
# through the top boundary at x = 0.78, which therefore carries both states;
# the final time is four flow-through times of the inflow (length / M1 = 0.5).
OBLIQUE_GAMMA = 1.4
OBLIQUE_LENGTH = 1.0
OBLIQUE_HEIGHT = 0.5
OBLIQUE_FINAL_TIME = 2.0


@dataclass(frozen=True, eq=False)
class ObliqueShockCase:
    solver: EulerSolver
    initial_state: np.ndarray
    final_time: float
    exact: object  # verification.ObliqueShock
    length: float
    height: float


def oblique_shock(nx: int = 100, ny: int = 50, *, flux: str, limiter: str, mach: float = 2.0,
                  wall_angle_deg: float = 10.0, length: float = OBLIQUE_LENGTH, height: float = OBLIQUE_HEIGHT,
                  final_time: float = OBLIQUE_FINAL_TIME, cfl: float = DEFAULT_CFL, precision: str = "fp64",
                  **solver_options) -> ObliqueShockCase:
    """Supersonic inflow (rho, u, v, p) = (1, M1, 0, 1/gamma) at the left,
    a slip wall along the inclined bottom, exact far-field states (ExactState)
    on the top and right, the upstream state everywhere at t = 0. Raises
    ValueError outside the attached weak-shock regime."""
    from .verification import ObliqueShock

    theta = np.radians(wall_angle_deg)
    exact = ObliqueShock(mach, theta, OBLIQUE_GAMMA)
    mesh = sheared_rectangle_mesh(nx, ny, theta, (0.0, length), (0.0, height))
    far = ExactState(exact.conserved, cell_average=exact.cell_average)
    bcs = {"left": FixedState.from_primitive(*exact.upstream, gamma=OBLIQUE_GAMMA), "bottom": SlipWall(),
           "top": far, "right": far}
    config = SolverConfig(flux=flux, limiter=limiter, gamma=OBLIQUE_GAMMA, cfl=cfl, precision=precision)
    solver = EulerSolver(mesh, bcs, config, **solver_options)
    upstream = np.array(FixedState.from_primitive(*exact.upstream, gamma=OBLIQUE_GAMMA).state)
    initial_state = np.broadcast_to(upstream, solver.state_shape).copy()
    return ObliqueShockCase(solver=solver, initial_state=initial_state, final_time=float(final_time), exact=exact,
                            length=float(length), height=float(height))
