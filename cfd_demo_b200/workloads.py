"""Seeded synthetic inputs of the 1M-triangle RK3 microbenchmark.

[0,1]^2 meshed as nx x nx quads, each split into 2 triangles (K = 2 nx^2; the
benchmark size nx = 724 gives K = 1,048,352), interior vertices jittered by
seeded uniform +-0.2h, every boundary tag a fixed state at the mean state
(rho, u, v, p) = (1, 0, 0, 1). Per-node fields are sums of 8 seeded random
Fourier modes, mapped affinely onto rho in [0.5, 1.5], u, v in [-0.5, 0.5]
and p in [0.5, 1.5]. flux = roe, limiter = unlimited (positivity still runs).

The same mesh and fields are built for the GPU solver (here), the CPU
oracle (the parity tests and the CPU baseline) and the benchmark, so each
sees bit-identical inputs.
"""

from __future__ import annotations

import math

import numpy as np

NX = 724
JITTER = 0.2
MESH_SEED = 20261203
FIELD_SEED = 7
GAMMA = 1.4
MEAN_STATE = (1.0, 0.0, 0.0, 1.0)
FIELD_RANGES = ((0.5, 1.5), (-0.5, 0.5), (-0.5, 0.5), (0.5, 1.5))


def fourier_field(x, y, rng, lo, hi, xp=np):
    """Sum of 8 random Fourier modes of the coordinates, mapped affinely
    onto [lo, hi]; ``xp`` is numpy or torch (device arrays)."""
    f = xp.zeros_like(x)
    for _ in range(8):
        kx, ky = rng.integers(1, 5, size=2)
        amp = rng.uniform(0.3, 1.0)
        ph = rng.uniform(0.0, 2 * math.pi)
        f = f + amp * xp.cos(2 * math.pi * (float(kx) * x + float(ky) * y) + ph)
    fmin, fmax = f.min(), f.max()
    return lo + (hi - lo) * (f - fmin) / (fmax - fmin)


def conserved_fields(x, y, xp=np):
    """(Np, K, 4) conserved state of the seeded Fourier fields at the node
    coordinates x, y (each (Np, K))."""
    rng = np.random.default_rng(FIELD_SEED)
    rho, u, v, p = (fourier_field(x, y, rng, lo, hi, xp) for lo, hi in FIELD_RANGES)
    e = p / (GAMMA - 1.0) + 0.5 * rho * (u * u + v * v)
    return xp.stack([rho, rho * u, rho * v, e], -1)


def microbenchmark_mesh(nx: int = NX):
    from .mesh import jittered_rectangle_mesh

    return jittered_rectangle_mesh(nx, nx, JITTER, MESH_SEED)


def microbenchmark_boundaries():
    from .boundary import FixedState

    mean = FixedState.from_primitive(*MEAN_STATE, GAMMA)
    return {t: mean for t in ("left", "right", "bottom", "top")}


def microbenchmark(nx: int = NX, precision: str = "fp32_mixed", device="cuda"):
    """(solver, initial state as a device (Np, K, 4) float64 tensor)."""
    import torch

    from .solver import EulerSolver, SolverConfig

    cfg = SolverConfig(flux="roe", limiter="unlimited", gamma=GAMMA, precision=precision)
    solver = EulerSolver(microbenchmark_mesh(nx), microbenchmark_boundaries(), cfg, device=device)
    x, y = solver.node_coordinates()
    q0 = conserved_fields(torch.as_tensor(x, device=device), torch.as_tensor(y, device=device), torch)
    return solver, q0.contiguous()
