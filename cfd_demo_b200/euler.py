"""Host-side conversions between primitive and conserved variables, for
building initial states and reading results (CFD-demo src/cfd_demo/euler.py:14-37).

Conserved variables are ordered (rho, rho u, rho v, E) along the last axis.
The solver's arithmetic runs in the CUDA kernels; these NumPy helpers only
prepare inputs and inspect outputs.
"""

from __future__ import annotations

import numpy as np

NUM_VARIABLES = 4


def primitive_to_conserved(rho, u, v, p, gamma: float) -> np.ndarray:
    rho, u, v, p = (np.asarray(a, dtype=np.float64) for a in (rho, u, v, p))
    energy = p / (gamma - 1.0) + 0.5 * rho * (u * u + v * v)
    return np.stack(np.broadcast_arrays(rho, rho * u, rho * v, energy), axis=-1)


def conserved_to_primitive(q, gamma: float):
    q = np.asarray(q, dtype=np.float64)
    rho = q[..., 0]
    u = q[..., 1] / rho
    v = q[..., 2] / rho
    p = (gamma - 1.0) * (q[..., 3] - 0.5 * (q[..., 1] * u + q[..., 2] * v))
    return rho, u, v, p


def pressure(q, gamma: float):
    return conserved_to_primitive(q, gamma)[3]


def sound_speed(rho, p, gamma: float):
    return np.sqrt(gamma * np.asarray(p) / np.asarray(rho))
