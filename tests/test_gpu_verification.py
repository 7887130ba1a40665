"""Verification of the Sod shock tube on the GPU: CFD-demo's ADR 0005
acceptance checks (tests/verification/test_sod_shock_tube.py of the
reference), run through the drop-in API.

The exact solution and the diagnostics are cfd_demo_b200.verification
(exact Riemann solver; L1 errors with elements cut at the exact wave
positions; shock position from column-averaged density), the thresholds are
the reference's: density L1 <= 0.03, shock within 0.02 of the exact position
(searched in 0.8 <= x <= 0.9), conservation defect <= 1e-8 against the
time-integrated boundary fluxes, and errors that drop under refinement.
"""

from __future__ import annotations

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

RESOLUTIONS = {"coarse": (100, 10), "fine": (200, 20)}
MAX_DENSITY_L1 = 0.03
MAX_SHOCK_ERROR = 0.02
MAX_CONSERVATION_DEFECT = 1e-8
SHOCK_WINDOW = (0.8, 0.9)


def _analyse(nx, ny, flux="rusanov", limiter="minmod", precision="fp64"):
    from cfd_demo_b200 import sod_shock_tube
    from cfd_demo_b200.cases import SOD_DISCONTINUITY, SOD_GAMMA, SOD_LEFT, SOD_RIGHT
    from cfd_demo_b200.verification import ExactRiemann, column_density, front_position, l1_errors

    case = sod_shock_tube(nx, ny, flux=flux, limiter=limiter, precision=precision)
    solver = case.solver
    initial = solver.integrate(case.initial_state)
    result = solver.run(case.initial_state, case.final_time)
    exact = ExactRiemann((SOD_LEFT[0], SOD_LEFT[1], SOD_LEFT[3]), (SOD_RIGHT[0], SOD_RIGHT[1], SOD_RIGHT[3]),
                         SOD_GAMMA, SOD_DISCONTINUITY)
    q = torch.from_numpy(result.state).cuda()
    errors = l1_errors(q, solver.mesh, exact, result.time, SOD_GAMMA)
    cols, faces = column_density(q, solver.mesh, nx)
    shock = front_position(cols, faces, SHOCK_WINDOW)
    defect = solver.integrate(result.state) - initial + result.boundary_flux_integral
    return {"case": case, "result": result, "errors": errors, "shock": shock, "defect": defect,
            "exact_shock": exact.wave_positions(result.time)["shock"]}


@pytest.fixture(scope="module")
def sod_runs(report):
    runs = {name: _analyse(*size) for name, size in RESOLUTIONS.items()}
    for name, r in runs.items():
        res = r["result"]
        report(f"verification Sod {name} {RESOLUTIONS[name]} rusanov/minmod: L1 "
               + ", ".join(f"{k} {v:.3e}" for k, v in r["errors"].items())
               + f"; shock {r['shock']:.5f} (exact {r['exact_shock']:.5f}); steps {res.steps}, "
               f"max troubled {res.max_troubled_cells}; conservation defect {np.abs(r['defect']).max():.2e}")
    return runs


@pytest.mark.parametrize("resolution", sorted(RESOLUTIONS))
def test_density_and_pressure_stay_positive(sod_runs, resolution):
    from cfd_demo_b200.cases import SOD_GAMMA

    res = sod_runs[resolution]["result"]
    q = res.state
    assert np.isfinite(q).all()
    rho = q[..., 0]
    p = (SOD_GAMMA - 1.0) * (q[..., 3] - 0.5 * (q[..., 1] ** 2 + q[..., 2] ** 2) / rho)
    assert rho.min() > 0.0 and p.min() > 0.0
    assert res.min_density > 0.0 and res.min_pressure > 0.0


@pytest.mark.parametrize("resolution", sorted(RESOLUTIONS))
def test_conservation_against_boundary_fluxes(sod_runs, resolution):
    r = sod_runs[resolution]
    assert np.abs(r["defect"]).max() <= MAX_CONSERVATION_DEFECT
    assert abs(r["result"].boundary_flux_integral[1]) > 1e-3  # the walls' net streamwise force
    assert r["result"].rejected_steps == 0


@pytest.mark.parametrize("resolution", sorted(RESOLUTIONS))
def test_density_error_and_shock_location(sod_runs, resolution):
    r = sod_runs[resolution]
    assert r["errors"]["density"] <= MAX_DENSITY_L1
    assert abs(r["shock"] - r["exact_shock"]) <= MAX_SHOCK_ERROR


def test_errors_decrease_under_refinement(sod_runs):
    assert sod_runs["fine"]["errors"]["density"] < sod_runs["coarse"]["errors"]["density"]
    for r in sod_runs.values():
        assert set(r["errors"]) == {"density", "pressure", "x velocity", "y velocity"}
        assert all(np.isfinite(v) for v in r["errors"].values())


def test_transverse_velocity_stays_small(sod_runs):
    e = sod_runs["fine"]["errors"]
    assert e["y velocity"] < e["x velocity"]


@pytest.mark.parametrize("flux,limiter", [("hllc", "van_leer"), ("roe", "superbee")])
def test_fp32_mixed_meets_the_same_acceptance_checks(flux, limiter, report):
    """The FP32-mixed form on the fine Sod tube: the same L1 and shock
    thresholds; mass, momentum and energy conserved to single-precision
    round-off (a few 1e-9 measured; a biased stage weight or a source in
    uniform regions shows up as 1e-5)."""
    r = _analyse(200, 20, flux=flux, limiter=limiter, precision="fp32_mixed")
    report(f"verification Sod 200x20 {flux}/{limiter} FP32-mixed: density L1 {r['errors']['density']:.3e}, "
           f"shock {r['shock']:.5f}; conservation defect {np.abs(r['defect']).max():.2e}")
    assert r["errors"]["density"] <= MAX_DENSITY_L1
    assert abs(r["shock"] - r["exact_shock"]) <= MAX_SHOCK_ERROR
    assert np.abs(r["defect"]).max() <= 1e-7
