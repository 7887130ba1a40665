"""Boundary conditions, applied only through the exterior state of the
interface flux (same interface as CFD-demo's src/cfd_demo/boundary.py)."""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

SLIP_WALL = 1
FIXED_STATE = 2
EXACT_STATE = 3


@dataclass(frozen=True)
class SlipWall:
    """Inviscid wall: the exterior state mirrors the interior trace with the
    normal momentum reversed."""

    kind: int = SLIP_WALL


@dataclass(frozen=True)
class FixedState:
    """Prescribed constant exterior state (rho, rho u, rho v, E)."""

    state: tuple[float, float, float, float]
    kind: int = FIXED_STATE

    def __post_init__(self) -> None:
        state = tuple(float(v) for v in self.state)
        if len(state) != 4 or not np.all(np.isfinite(state)):
            raise ValueError("FixedState needs four finite conserved values.")
        object.__setattr__(self, "state", state)

    @classmethod
    def from_primitive(cls, rho: float, u: float, v: float, p: float, gamma: float) -> "FixedState":
        energy = p / (gamma - 1.0) + 0.5 * rho * (u * u + v * v)
        return cls((rho, rho * u, rho * v, energy))


@dataclass(frozen=True, eq=False)
class ExactState:
    """Exterior states from a known solution (CFD-demo's proposed ADR 0012,
    docs/adr/0012-...:32-46): `function(x, y)` maps arrays of physical
    coordinates to conserved states of shape x.shape + (4,). It is evaluated
    once, when the solver is built, at every face node of the tagged faces
    (per-node exterior states of the interface flux), and its cell average
    over each boundary element reflected across the boundary face is the
    ghost average of the troubled-cell limiter: `cell_average(corners)`
    ((n, 3, 2) triangles -> (n, 4)) when given, else the mean over the
    centroids of 32 x 32 equal sub-triangles. For verification with an
    analytic solution, not a general outflow condition."""

    function: object
    cell_average: object = None
    kind: int = EXACT_STATE

    def __post_init__(self) -> None:
        if not callable(self.function):
            raise ValueError("ExactState needs a callable function(x, y) -> conserved states.")
        if self.cell_average is not None and not callable(self.cell_average):
            raise ValueError("ExactState cell_average must be callable (or None).")

    def states(self, x: np.ndarray, y: np.ndarray) -> np.ndarray:
        x, y = np.asarray(x, dtype=np.float64), np.asarray(y, dtype=np.float64)
        q = np.asarray(self.function(x, y), dtype=np.float64)
        if q.shape != x.shape + (4,) or not np.all(np.isfinite(q)):
            raise ValueError("ExactState function must return finite conserved states of shape x.shape + (4,).")
        return q


BoundaryCondition = SlipWall | FixedState | ExactState
