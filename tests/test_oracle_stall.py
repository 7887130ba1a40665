"""The reference algorithm (the oracle, on the CPU) on instance 25 of the
seeded Riemann family of the batching benchmark: a near-vacuum forms at
t ~ 0.0027 and the CFL step collapses, so this instance cannot reach the
benchmark's t = 0.15. The GPU batch shows the same stall
(tests/test_gpu_batch.py follows the oracle's step sizes through it)."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.slow


def test_reference_algorithm_stalls_on_instance_25():
    import oracle
    from oracle.physics import FixedState, SlipWall

    from cfd_demo_b200.batch import riemann_batch

    case = riemann_batch(256, seed=0)[25]
    m = case.mesh
    om = oracle.mesh.TriangleMesh(np.array(m.vertices), np.array(m.elements),
                                  {k: np.array(v) for k, v in m.boundary_edges.items()})
    bcs = {t: (FixedState(tuple(b.state)) if b.kind == 2 else SlipWall()) for t, b in case.boundary_conditions.items()}
    s = oracle.OracleSolver(om, bcs, flux="hllc", limiter="superbee", gamma=1.4)
    q, dts, t = case.initial_state, [], 0.0
    for _ in range(80):
        dt = s.time_step(q)
        q, rep = s.step(q, dt)
        assert rep.admissible
        dts.append(dt)
        t += dt
    assert t < 0.003
    assert dts[-1] < dts[0] / 50
    assert rep.min_density < 1e-3
