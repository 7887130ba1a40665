"""Pin the CPU oracle against golden vectors generated by the reference's own
source (tests/golden/make_golden.py). CPU only.

Tolerances: the oracle and the reference both evaluate in NumPy float64 but in
different operation orders, so values agree to round-off (1e-12 relative to
the field's scale). Troubled-cell flags and counts must agree exactly.
"""

from __future__ import annotations

import numpy as np
import pytest

import oracle
from oracle.mesh import TriangleMesh
from oracle.physics import FixedState, SlipWall
from tests.golden_io import FLUXES, GAMMA, LIMITERS, boundary_specs, case_prefixes, load, mesh_parts, unpack_flags


def oracle_solver(data, prefix, flux="rusanov", limiter="minmod"):
    v, e, edges = mesh_parts(data, prefix)
    bcs = {tag: (SlipWall() if kind == 1 else FixedState(state)) for tag, (kind, state) in boundary_specs(data, prefix).items()}
    return oracle.OracleSolver(TriangleMesh(v, e, edges), bcs, flux=flux, limiter=limiter, gamma=GAMMA)


def close(a, b, rel=1e-12):
    a, b = np.asarray(a), np.asarray(b)
    scale = max(float(np.abs(b).max()), 1e-300)
    return float(np.abs(a - b).max()) <= rel * scale


def test_reference_element_tables():
    g = load("element")
    ref = oracle.build_reference_triangle(4)
    for key in ("r", "s", "dr", "ds", "lift", "cell_weights", "face_weights", "p1_midpoint", "linear_midpoint_basis"):
        assert np.allclose(getattr(ref, key), g[key], rtol=0, atol=1e-12), key
    assert np.array_equal(ref.face_nodes, g["face_nodes"])
    assert np.array_equal(ref.face_midpoint_nodes, g["face_midpoint_nodes"])


def test_pointwise_fluxes_and_phi():
    g = load("pointwise")
    qm, qp, nx, ny = g["q_minus"], g["q_plus"], g["nx"], g["ny"]
    for name in FLUXES:
        assert np.allclose(oracle.get_interface_flux(name)(qm, qp, nx, ny, GAMMA), g[f"flux/{name}"], rtol=1e-13, atol=1e-13), name
    f, gg = oracle.cartesian_fluxes(qm, GAMMA)
    assert np.allclose(f, g["cartesian/f"], rtol=1e-14, atol=0)
    assert np.allclose(gg, g["cartesian/g"], rtol=1e-14, atol=0)
    for name in LIMITERS:
        assert np.array_equal(oracle.get_limiter_function(name)(g["phi/r"]), g[f"phi/{name}"]), name


@pytest.mark.parametrize("prefix", case_prefixes(load("rhs")))
@pytest.mark.parametrize("flux", FLUXES)
def test_rhs_matches_reference(prefix, flux):
    g = load("rhs")
    s = oracle_solver(g, prefix, flux=flux)
    rhs, bflux = s.rhs(g[f"{prefix}/q"])
    ref_rhs = g[f"{prefix}/rhs/{flux}"]
    scale = max(np.abs(ref_rhs).max(), 1.0)
    assert np.abs(rhs - ref_rhs).max() <= 1e-12 * scale
    assert np.abs(bflux - g[f"{prefix}/bflux/{flux}"]).max() <= 1e-12 * max(np.abs(g[f"{prefix}/bflux/{flux}"]).max(), 1.0)


@pytest.mark.parametrize("prefix", case_prefixes(load("limit")))
@pytest.mark.parametrize("limiter", LIMITERS)
def test_limit_matches_reference(prefix, limiter):
    g = load("limit")
    s = oracle_solver(g, prefix, limiter=limiter)
    q = g[f"{prefix}/q"]
    limited, avg, count, flags = s.apply_limiters(q)
    assert close(limited, g[f"{prefix}/limited/{limiter}"])
    assert count == int(g[f"{prefix}/count/{limiter}"])
    if limiter != "unlimited":
        assert np.array_equal(flags, g[f"{prefix}/troubled/{limiter}"])
    assert close(s.cell_averages(q), g[f"{prefix}/averages"])
    assert close(s.integrate(q), g[f"{prefix}/integral"])


@pytest.mark.parametrize("flux", FLUXES)
@pytest.mark.parametrize("limiter", LIMITERS)
def test_step_matches_reference(flux, limiter):
    g = load("step")
    s = oracle_solver(g, "mesh", flux=flux, limiter=limiter)
    key = f"{flux}/{limiter}"
    dt = s.time_step(g["q"])
    assert dt == pytest.approx(float(g[f"{key}/dt"]), rel=1e-13)
    qn, rep = s.step(g["q"], float(g[f"{key}/dt"]))
    assert close(qn, g[f"{key}/q_new"], rel=1e-11)
    assert np.allclose(rep.boundary_flux, g[f"{key}/boundary_flux"], rtol=1e-11, atol=1e-15)
    assert rep.admissible == bool(g[f"{key}/admissible"])
    assert rep.min_density == pytest.approx(float(g[f"{key}/min_density"]), rel=1e-11)
    assert rep.min_pressure == pytest.approx(float(g[f"{key}/min_pressure"]), rel=1e-9, abs=1e-20)
    assert rep.troubled_cells == int(g[f"{key}/troubled_cells"])


def test_short_sod_run_matches_reference():
    g = load("sod_short")
    s = oracle.OracleSolver(oracle.rectangle_mesh(20, 2), {
        "left": FixedState.from_primitive(1.0, 0.0, 0.0, 1.0, GAMMA),
        "right": FixedState.from_primitive(0.125, 0.0, 0.0, 0.1, GAMMA),
        "bottom": SlipWall(), "top": SlipWall()}, flux="rusanov", limiter="minmod", gamma=GAMMA)
    trace = []
    flags = []
    res = s.run(g["initial_state"], 0.01, trace=trace)
    assert res.steps == int(g["steps"]) and res.rejected_steps == int(g["rejected_steps"])
    assert res.time == float(g["time"])
    assert np.allclose([t[0] for t in trace], g["dt"], rtol=1e-12, atol=0)
    assert [t[1].troubled_cells for t in trace] == list(g["stage_troubled"].max(axis=1))
    assert close(res.state, g["state"], rel=1e-11)
    assert np.allclose(res.boundary_flux_integral, g["boundary_flux_integral"], rtol=1e-10, atol=1e-15)
    # stage-by-stage troubled flags of every step
    ref_flags = unpack_flags(g)
    q = g["initial_state"]
    for n, (dt, _) in enumerate(trace[: ref_flags.shape[0]]):
        rec = []
        q, _ = s.step(q, dt, record=rec)
        assert np.array_equal(np.stack(rec), ref_flags[n]), f"step {n}"
