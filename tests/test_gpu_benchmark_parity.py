"""Parity on the benchmark configuration itself: the 1M-triangle workload
(724 x 724 quads x 2 triangles, K = 1,048,352, jitter +-0.2h, 8-mode Fourier
fields, roe/unlimited, fixed-state boundaries), the FP64 CUDA path against the
CPU oracle on bit-identical inputs:

  * one RHS (dg.py:140-165): <= 1e-12 relative per node, boundary flux 1e-12;
  * the CFL step (time_integration.py:37-41): <= 1e-13 relative;
  * one SSP-RK3 step (time_integration.py:44-84): <= 1e-11 relative per node,
    report fields as the oracle's;

and the FP32-mixed form against that FP64 step: L1 / Linf density difference
and the mass / energy conservation defect of each form. These sizes exercise
the index arithmetic at ld ~ 1M and the jittered-mesh face pairing. The oracle
needs about two minutes of CPU time here.
"""

from __future__ import annotations

import numpy as np
import pytest

from tests.gpu_helpers import rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def bench_case():
    import oracle
    from cfd_demo_b200 import EulerSolver, SolverConfig
    from cfd_demo_b200.workloads import GAMMA, conserved_fields, microbenchmark_boundaries, microbenchmark_mesh
    from oracle.physics import FixedState

    mesh = microbenchmark_mesh()
    s64 = EulerSolver(mesh, microbenchmark_boundaries(), SolverConfig(flux="roe", limiter="unlimited", gamma=GAMMA))
    x, y = s64.node_coordinates()
    q0 = np.ascontiguousarray(conserved_fields(x, y, np))
    omesh = oracle.mesh.TriangleMesh(np.array(mesh.vertices), np.array(mesh.elements),
                                     {k: np.array(v) for k, v in mesh.boundary_edges.items()})
    mean = FixedState.from_primitive(1.0, 0.0, 0.0, 1.0, GAMMA)
    osolver = oracle.OracleSolver(omesh, {t: mean for t in ("left", "right", "bottom", "top")}, flux="roe",
                                  limiter="unlimited", gamma=GAMMA)
    ox, oy = osolver.node_coordinates()
    assert np.array_equal(ox, x) and np.array_equal(oy, y)
    return s64, osolver, q0


def test_rhs_matches_the_oracle_at_benchmark_size(bench_case, report):
    s64, osolver, q0 = bench_case
    assert s64.mesh.num_elements == 1_048_352
    rhs, bflux = s64.rhs(q0)
    orhs, obflux = osolver.rhs(q0)
    err = rel_err(rhs, orhs)
    report(f"1M-triangle benchmark mesh (K={s64.mesh.num_elements}), FP64 RHS vs oracle: rel err {err:.2e}")
    assert err <= 1e-12
    assert np.abs(bflux - obflux).max() <= 1e-12 * max(np.abs(obflux).max(), 1.0)


def test_step_matches_the_oracle_at_benchmark_size(bench_case, report):
    s64, osolver, q0 = bench_case
    dt = s64.time_step(q0)
    odt = osolver.time_step(q0)
    assert dt == pytest.approx(odt, rel=1e-13)
    q1, rep = s64.step(q0, odt)
    oq1, orep = osolver.step(q0, odt)
    err = rel_err(q1, oq1)
    report(f"1M-triangle benchmark mesh, FP64 RK3 step vs oracle: rel err {err:.2e}, dt {dt:.17g} "
           f"(oracle {odt:.17g})")
    assert err <= 1e-11
    assert rep.admissible and orep.admissible
    np.testing.assert_allclose(rep.boundary_flux, orep.boundary_flux, rtol=1e-11, atol=1e-15)
    assert rep.min_density == pytest.approx(orep.min_density, rel=1e-12)
    assert rep.min_pressure == pytest.approx(orep.min_pressure, rel=1e-12)


def test_fp32_mixed_against_fp64_at_benchmark_size(bench_case, report):
    """Ten steps of each form from the same state with the same step sizes
    (the FP64 run's CFL steps): the FP32-mixed density
    against the FP64 one (L1 domain-averaged, Linf), and each form's mass and
    energy defect (final - initial integral + time-integrated boundary flux)."""
    s64, _, q0 = bench_case
    s32 = s64.with_precision("fp32_mixed")
    out = {}
    dts = []
    for name, s in (("fp64", s64), ("fp32_mixed", s32)):
        q = q0
        flux = np.zeros(4)
        for n in range(10):
            if name == "fp64":  # both forms take the FP64 run's CFL steps
                dts.append(s.time_step(q))
            q, rep = s.step(q, dts[n])
            assert rep.admissible
            flux += rep.boundary_flux
        defect = s64.integrate(q) - s64.integrate(q0) + flux
        out[name] = (q, defect)
    d = np.abs(out["fp32_mixed"][0][..., 0] - out["fp64"][0][..., 0])
    w = s64.reference.cell_weights
    jac = np.asarray(s64.geometry.jacobian)
    l1 = float(np.einsum("i,ik,k->", w, d, jac) / np.einsum("i,k->", w, jac))
    linf = float(d.max())
    m64, e64 = out["fp64"][1][0], out["fp64"][1][3]
    m32, e32 = out["fp32_mixed"][1][0], out["fp32_mixed"][1][3]
    report(f"1M-triangle benchmark mesh, 10 CFL steps FP32-mixed vs FP64: L1(rho) {l1:.2e}, Linf(rho) {linf:.2e}; "
           f"mass / energy defect FP64 {m64:.1e} / {e64:.1e}, FP32-mixed {m32:.1e} / {e32:.1e}")
    assert l1 <= 1e-5
    assert linf <= 1e-3
    assert abs(m64) <= 1e-13 and abs(e64) <= 1e-12
    assert abs(m32) <= 1e-6 and abs(e32) <= 1e-5
