"""Batched instances (meshes of uneven size in one launch) against the same
problems solved one at a time: identical step counts, end times and states."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision,variant", [("fp64", 0), ("fp64", 2), ("fp32_mixed", 0), ("fp32_mixed", 3)])
def test_batch_matches_single_instance_runs(precision, variant):
    from cfd_demo_b200 import EulerSolver, SolverConfig
    from cfd_demo_b200.batch import BatchedEulerSolver, riemann_batch

    cases = riemann_batch(count=6, seed=3, nx_range=(10, 40))
    cfg = SolverConfig(flux="hllc", limiter="superbee", gamma=1.4, precision=precision)
    batch = BatchedEulerSolver(cases, cfg, variant=variant)
    results = batch.run(final_time=0.02)
    tol = 1e-12 if precision == "fp64" else 1e-6
    for case, res in zip(cases, results):
        single = EulerSolver(case.mesh, case.boundary_conditions, cfg, variant=variant)
        ref = single.run(case.initial_state, 0.02)
        assert res.steps == ref.steps and res.rejected_steps == ref.rejected_steps
        assert res.time == ref.time
        assert res.max_troubled_cells == ref.max_troubled_cells
        scale = np.maximum(np.abs(ref.state).reshape(-1, 4).max(axis=0), 1e-300)
        assert float((np.abs(res.state - ref.state) / scale).max()) <= tol
        np.testing.assert_allclose(res.boundary_flux_integral, ref.boundary_flux_integral, rtol=1e-9, atol=1e-12)


def test_batch_instances_finish_at_their_own_times():
    from cfd_demo_b200 import SolverConfig
    from cfd_demo_b200.batch import BatchedEulerSolver, riemann_batch

    cases = riemann_batch(count=5, seed=1, nx_range=(8, 24))
    batch = BatchedEulerSolver(cases, SolverConfig(flux="rusanov", limiter="minmod", gamma=1.4))
    times = np.array([0.005, 0.01, 0.0, 0.02, 0.015])
    res = batch.run(final_time=times)
    assert [r.time for r in res] == pytest.approx(list(times), abs=0.0)
    assert res[2].steps == 0
    for r, case in zip(res, cases):
        assert np.all(np.isfinite(r.state))
