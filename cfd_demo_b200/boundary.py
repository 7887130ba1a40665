"""Boundary conditions, applied only through the exterior state of the
interface flux (same interface as CFD-demo's src/cfd_demo/boundary.py)."""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

SLIP_WALL = 1
FIXED_STATE = 2


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


BoundaryCondition = SlipWall | FixedState
