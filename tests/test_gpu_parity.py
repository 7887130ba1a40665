"""GPU parity of the sm_100a kernels (through the C ABI) against golden vectors
made by the reference's own source and against the CPU oracle.

Tolerances (plain FP64 form), "relative" = |gpu - ref| / max |ref| of the same
conserved variable over the mesh:
  * one RHS evaluation:                 1e-12
  * limiters, one RK3 step:             1e-12 / 1e-11
  * the 20x2 Sod run:                   1e-10 (final state), identical step
                                        counts and troubled-cell maxima
  * the 100x10 Sod run:                 tests/test_gpu_flags.py
  * troubled-cell counts and flags:     exact
  * pointwise interface fluxes:         1e-13 relative + 1e-13 absolute
  * phi(r):                             bit-exact
"""

from __future__ import annotations

import numpy as np
import pytest

from tests.golden_io import FLUXES, GAMMA, LIMITERS, case_prefixes, load
from tests.gpu_helpers import make_solver, rel_err

pytestmark = pytest.mark.gpu


def test_pointwise_fluxes_match_reference():
    from cfd_demo_b200 import get_interface_flux

    g = load("pointwise")
    for name in FLUXES:
        out = get_interface_flux(name)(g["q_minus"], g["q_plus"], g["nx"], g["ny"], GAMMA)
        np.testing.assert_allclose(out, g[f"flux/{name}"], rtol=1e-13, atol=1e-13, err_msg=name)


def test_phi_bit_exact():
    from cfd_demo_b200 import get_limiter_function

    g = load("pointwise")
    for name in LIMITERS:
        assert np.array_equal(get_limiter_function(name)(g["phi/r"]), g[f"phi/{name}"]), name


@pytest.mark.parametrize("prefix", case_prefixes(load("rhs")))
@pytest.mark.parametrize("flux", FLUXES)
@pytest.mark.parametrize("variant", [0, 2, 3, 10])
def test_rhs_matches_reference(prefix, flux, variant):
    g = load("rhs")
    s = make_solver(g, prefix, flux=flux, variant=variant)
    rhs, bflux = s.rhs(g[f"{prefix}/q"])
    ref = g[f"{prefix}/rhs/{flux}"]
    if prefix == "freestream":
        assert np.abs(rhs).max() < 1e-11
    else:
        assert rel_err(rhs, ref) <= 1e-12
    rb = g[f"{prefix}/bflux/{flux}"]
    assert np.abs(bflux - rb).max() <= 1e-12 * max(np.abs(rb).max(), 1.0)


@pytest.mark.parametrize("prefix", case_prefixes(load("limit")))
@pytest.mark.parametrize("limiter", LIMITERS)
def test_limit_matches_reference(prefix, limiter):
    g = load("limit")
    s = make_solver(g, prefix, limiter=limiter)
    q = g[f"{prefix}/q"]
    limited, count = s.limit_with_count(q)
    assert rel_err(limited, g[f"{prefix}/limited/{limiter}"]) <= 1e-12
    assert count == int(g[f"{prefix}/count/{limiter}"])
    if limiter != "unlimited":
        # the elements the limiter changed are exactly the troubled ones or
        # the ones the positivity limiter touched
        flags = g[f"{prefix}/troubled/{limiter}"]
        changed = np.any(np.abs(limited - q) > 0, axis=(0, 2))
        assert np.all(changed[flags]) or prefix == "positivity"
    assert np.abs(s.cell_averages(q) - g[f"{prefix}/averages"]).max() <= 1e-13 * np.abs(g[f"{prefix}/averages"]).max()
    np.testing.assert_allclose(s.integrate(q), g[f"{prefix}/integral"], rtol=1e-12, atol=1e-15)


def test_positivity_floor_is_met_exactly():
    """The reference's own acceptance (test_limiting_and_time.py:91-109):
    every node ends at >= 1e-13 (1 - 1e-9) in density and pressure."""
    from cfd_demo_b200.euler import conserved_to_primitive

    g = load("limit")
    s = make_solver(g, "positivity", limiter="unlimited")
    q = g["positivity/q"]
    limited = s.limit(q)
    rho, _, _, p = conserved_to_primitive(limited, GAMMA)
    assert rho.min() >= 1e-13 * (1.0 - 1e-9)
    assert p.min() >= 1e-13 * (1.0 - 1e-9)
    assert np.abs(s.cell_averages(limited) - s.cell_averages(q)).max() < 1e-12


@pytest.mark.parametrize("flux", FLUXES)
@pytest.mark.parametrize("limiter", LIMITERS)
@pytest.mark.parametrize("variant", [0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14])
def test_step_matches_reference(flux, limiter, variant):
    g = load("step")
    s = make_solver(g, "mesh", flux=flux, limiter=limiter, variant=variant)
    key = f"{flux}/{limiter}"
    assert s.time_step(g["q"]) == pytest.approx(float(g[f"{key}/dt"]), rel=1e-13)
    qn, rep = s.step(g["q"], float(g[f"{key}/dt"]))
    assert rel_err(qn, g[f"{key}/q_new"]) <= 1e-11
    np.testing.assert_allclose(rep.boundary_flux, g[f"{key}/boundary_flux"], rtol=1e-11, atol=1e-15)
    assert rep.admissible == bool(g[f"{key}/admissible"])
    assert rep.min_density == pytest.approx(float(g[f"{key}/min_density"]), rel=1e-11)
    assert rep.min_pressure == pytest.approx(float(g[f"{key}/min_pressure"]), rel=1e-9, abs=1e-18)
    assert rep.troubled_cells == int(g[f"{key}/troubled_cells"])


def _sod_like(nx, ny, flux="rusanov", limiter="minmod"):
    from cfd_demo_b200 import EulerSolver, SolverConfig, rectangle_mesh
    from cfd_demo_b200.cases import sod_boundaries

    return EulerSolver(rectangle_mesh(nx, ny), sod_boundaries(), SolverConfig(flux=flux, limiter=limiter, gamma=GAMMA))


@pytest.mark.parametrize("graph", [True, False])
def test_short_sod_run_matches_reference(graph):
    g = load("sod_short")
    s = _sod_like(20, 2)
    res = s.run(g["initial_state"], 0.01, graph=graph)
    assert res.steps == int(g["steps"]) and res.rejected_steps == int(g["rejected_steps"])
    assert res.time == float(g["time"])
    assert res.max_troubled_cells == int(g["max_troubled_cells"])
    assert rel_err(res.state, g["state"]) <= 1e-10
    np.testing.assert_allclose(res.boundary_flux_integral, g["boundary_flux_integral"], rtol=1e-10, atol=1e-14)
    assert res.min_density == pytest.approx(float(g["min_density"]), rel=1e-10)


def test_short_sod_stage_troubled_counts_match_per_step():
    """March the golden dt sequence step by step: per-step troubled maxima
    must match exactly (the flags are decided in the reference's op order)."""
    g = load("sod_short")
    s = _sod_like(20, 2)
    q = g["initial_state"]
    for n, dt in enumerate(g["dt"]):
        q, rep = s.step(q, float(dt))
        assert rep.troubled_cells == int(g["stage_troubled"][n].max()), f"step {n}"
        assert rep.admissible


@pytest.mark.parametrize("variant", [0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14])
def test_fp32_mixed_step_tracks_fp64(variant):
    """The FP32-mixed form against the plain form on the step fixture: one RK3
    step agrees to FP32 accuracy (1e-5 of each variable's scale)."""
    g = load("step")
    s64 = make_solver(g, "mesh", flux="roe", limiter="unlimited")
    s32 = make_solver(g, "mesh", flux="roe", limiter="unlimited", precision="fp32_mixed", variant=variant)
    dt = float(g["roe/unlimited/dt"])
    q64, r64 = s64.step(g["q"], dt)
    q32, r32 = s32.step(g["q"], dt)
    assert rel_err(q32, q64) <= 1e-5
    assert r32.admissible and r64.admissible


@pytest.mark.parametrize("precision", ["fp64", "fp32_mixed"])
@pytest.mark.parametrize("limiter", ["minmod", "superbee", "unlimited"])
def test_two_pass_limiter_is_bitwise_the_one_pass_limiter(limiter, precision):
    """The limiter's two-pass form (detection scan over every element, then
    the rewrite of the listed ones) gives the one-pass kernel's results bit
    for bit: a Sod run (troubled cells and the positivity floor) and one
    cfd_limit call."""
    from cfd_demo_b200 import sod_shock_tube

    case = sod_shock_tube(60, 6, flux="hllc", limiter=limiter, precision=precision)
    s = case.solver
    assert s.native.limit_list
    two = s.run(case.initial_state, 0.03)
    lim_two, count_two = s.limit_with_count(two.state)
    s.native.limit_list = None
    s._graphs.clear()
    one = s.run(case.initial_state, 0.03)
    lim_one, count_one = s.limit_with_count(two.state)
    assert np.array_equal(one.state, two.state), np.abs(one.state - two.state).max()
    assert (one.steps, one.max_troubled_cells, one.rejected_steps) == (two.steps, two.max_troubled_cells,
                                                                        two.rejected_steps)
    assert one.min_density == two.min_density and one.min_pressure == two.min_pressure
    # the boundary-flux integral is a sum of floating-point atomics: its last
    # bits depend on their order, in either form
    assert np.allclose(one.boundary_flux_integral, two.boundary_flux_integral, rtol=1e-12, atol=1e-15)
    assert np.array_equal(lim_one, lim_two), np.abs(lim_one - lim_two).max()
    assert count_one == count_two


@pytest.mark.parametrize("flux", FLUXES)
@pytest.mark.parametrize("scalar,packed", [(6, 3), (7, 5)])
def test_packed_fp32_contractions_are_bitwise_the_scalar_ones(flux, scalar, packed):
    """The tiled shapes issue the FP32 [Dr|Ds] and LIFT contractions as packed
    FP32x2 FMAs; variants 6 / 7 are shapes 3 / 5 with scalar FMAs. Each packed
    lane rounds like a scalar FMA, so a Sod run and one RHS agree bit for bit."""
    from cfd_demo_b200 import sod_shock_tube

    out = {}
    for v in (scalar, packed):
        case = sod_shock_tube(60, 6, flux=flux, limiter="minmod", precision="fp32_mixed")
        case.solver.set_variant(v)
        res = case.solver.run(case.initial_state, 0.02)
        rhs, _ = case.solver.rhs(res.state)
        out[v] = (res, rhs)
    (a, ra), (b, rb) = out[scalar], out[packed]
    assert a.steps == b.steps and a.max_troubled_cells == b.max_troubled_cells
    assert np.array_equal(a.state, b.state), np.abs(a.state - b.state).max()
    assert np.array_equal(ra, rb), np.abs(ra - rb).max()
