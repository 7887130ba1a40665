"""Helpers shared by the GPU tests: build cfd_demo_b200 solvers from the golden
fixtures' meshes and compare fields with explicit tolerances."""

from __future__ import annotations

import numpy as np

from tests.golden_io import GAMMA, boundary_specs, mesh_parts


def make_solver(data, prefix, flux="rusanov", limiter="minmod", precision="fp64", **kw):
    from cfd_demo_b200 import EulerSolver, FixedState, SlipWall, SolverConfig, TriangleMesh

    v, e, edges = mesh_parts(data, prefix)
    bcs = {t: (SlipWall() if k == 1 else FixedState(s)) for t, (k, s) in boundary_specs(data, prefix).items()}
    cfg = SolverConfig(flux=flux, limiter=limiter, gamma=GAMMA, precision=precision)
    return EulerSolver(TriangleMesh(v, e, edges), bcs, cfg, **kw)


def rel_err(a, b, axis_scale=True) -> float:
    """max |a - b| / scale, scale = max |b| per conserved variable (last axis),
    floored at 1e-300. This is the "relative per node" metric of the parity
    tests: every node's error measured against its field's magnitude."""
    a, b = np.asarray(a), np.asarray(b)
    if axis_scale and b.ndim >= 1 and b.shape[-1] == 4:
        scale = np.maximum(np.abs(b).reshape(-1, 4).max(axis=0), 1e-300)
        return float((np.abs(a - b) / scale).max())
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))
