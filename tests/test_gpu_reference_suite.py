"""The reference's unit-test suite (tests/unit/test_dg_operator.py,
test_limiting_and_time.py, test_physics.py of CFD-demo), restated against the
B200 solver: the same properties with the same thresholds, run through the
sm_100a kernels."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GAMMA = 1.4
FREE_STREAM = (1.2, 0.4, -0.3, 0.9)
FLUXES = ("hllc", "roe", "rusanov")
STATES = ((1.0, 0.0, 0.0, 1.0), (0.125, 0.0, 0.0, 0.1), (1.3, 0.7, -0.4, 2.1), (0.4, -1.2, 0.9, 0.3))


def perturbed_mesh(nx, ny, amplitude=0.25, seed=0):
    from cfd_demo_b200 import TriangleMesh, rectangle_mesh

    m = rectangle_mesh(nx, ny)
    v = np.array(m.vertices)
    inside = np.all((v > 1e-12) & (v < 1.0 - 1e-12), axis=1)
    d = np.random.default_rng(seed).uniform(-1.0, 1.0, size=v.shape)
    v[inside] += amplitude * d[inside] / np.array([nx, ny])
    return TriangleMesh(vertices=v, elements=m.elements, boundary_edges=m.boundary_edges)


def make_solver(mesh, conditions, flux="rusanov", limiter="minmod", **cfg):
    from cfd_demo_b200 import EulerSolver, SolverConfig

    return EulerSolver(mesh, conditions, SolverConfig(flux=flux, limiter=limiter, gamma=GAMMA, **cfg))


def uniform_state(solver, primitive):
    from cfd_demo_b200.euler import primitive_to_conserved

    return np.broadcast_to(primitive_to_conserved(*primitive, GAMMA), solver.state_shape).copy()


def fixed_all(primitive):
    from cfd_demo_b200 import FixedState

    c = FixedState.from_primitive(*primitive, GAMMA)
    return {t: c for t in ("left", "right", "bottom", "top")}


def walls_all():
    from cfd_demo_b200 import SlipWall

    return {t: SlipWall() for t in ("left", "right", "bottom", "top")}


# ---- DG operator (test_dg_operator.py) -------------------------------------------
@pytest.mark.parametrize("flux", FLUXES)
def test_free_stream_is_preserved_on_a_distorted_mesh(flux):
    s = make_solver(perturbed_mesh(6, 5), fixed_all(FREE_STREAM), flux=flux)
    rhs, _ = s.rhs(uniform_state(s, FREE_STREAM))
    assert np.abs(rhs).max() < 1e-11


@pytest.mark.parametrize("flux", FLUXES)
def test_fp32_mixed_free_stream_is_exact(flux):
    """In the FP32-mixed form a uniform state has an exactly zero right-hand
    side: the volume term differentiates F~ - F~(node 0) and equal traces give
    F(q).n exactly, so the rounded tables and metric leave no source in
    uniform regions (a source there accumulated into a steady mass and energy
    drift). A time step then changes the state only by the single-precision
    rounding of the stage-2 weights 0.75 / 0.25."""
    s = make_solver(perturbed_mesh(6, 5), fixed_all(FREE_STREAM), flux=flux, precision="fp32_mixed")
    q = uniform_state(s, FREE_STREAM).astype(np.float32).astype(np.float64)  # representable in float
    rhs, _ = s.rhs(q)
    assert np.all(rhs == 0.0), np.abs(rhs).max()
    advanced, rep = s.step(q, s.time_step(q))
    assert np.abs(advanced - q).max() <= 2.5e-7 * np.abs(q).max() and rep.admissible


def test_free_stream_survives_limiting_and_a_time_step():
    s = make_solver(perturbed_mesh(6, 5), fixed_all(FREE_STREAM))
    q = uniform_state(s, FREE_STREAM)
    assert np.abs(s.limit(q) - q).max() < 1e-13
    advanced, rep = s.step(q, s.time_step(q))
    assert np.abs(advanced - q).max() < 1e-11
    assert rep.admissible and rep.troubled_cells == 0


def test_slip_walls_keep_a_closed_box_at_rest():
    s = make_solver(perturbed_mesh(5, 4), walls_all())
    rhs, bflux = s.rhs(uniform_state(s, (1.0, 0.0, 0.0, 1.0)))
    assert np.abs(rhs).max() < 1e-12
    assert np.abs(bflux).max() < 1e-12


def test_slip_wall_reflects_the_normal_momentum():
    from cfd_demo_b200 import rectangle_mesh

    s = make_solver(rectangle_mesh(4, 4), walls_all(), flux="rusanov")
    rho, u, p = 1.0, 0.5, 1.0
    _, bflux = s.rhs(uniform_state(s, (rho, u, 0.0, p)))
    assert np.abs(bflux[[0, 2, 3]]).max() < 1e-12
    assert bflux[1] == pytest.approx(2.0 * (abs(u) + np.sqrt(GAMMA * p / rho)) * rho * u, abs=1e-12)


@pytest.mark.parametrize("flux", FLUXES)
def test_discrete_conservation_identity(flux):
    from cfd_demo_b200.euler import primitive_to_conserved

    s = make_solver(perturbed_mesh(5, 4, seed=3), fixed_all(FREE_STREAM), flux=flux)
    prim = np.random.default_rng(11).uniform([0.5, -0.4, -0.4, 0.5], [1.5, 0.4, 0.4, 1.5], size=s.state_shape[:2] + (4,))
    q = primitive_to_conserved(*(prim[..., k] for k in range(4)), GAMMA)
    rhs, bflux = s.rhs(q)
    assert np.abs(s.integrate(rhs) + bflux).max() < 1e-12
    assert np.abs(bflux).max() > 1e-3


def test_integrate_and_cell_averages_agree():
    from cfd_demo_b200.euler import primitive_to_conserved

    s = make_solver(perturbed_mesh(4, 3), fixed_all(FREE_STREAM))
    q = uniform_state(s, FREE_STREAM)
    cons = primitive_to_conserved(*FREE_STREAM, GAMMA)
    assert np.allclose(s.cell_averages(q), cons)
    assert np.allclose(s.integrate(q), cons)
    assert np.allclose((s.cell_averages(q) * s.geometry.area[:, None]).sum(axis=0), s.integrate(q))


def _smooth_primitives(x, y):
    tp = 2.0 * np.pi
    return (1.0 + 0.2 * np.sin(tp * x) * np.sin(tp * y), 0.3 + 0.1 * np.cos(tp * x) * np.sin(tp * y),
            -0.2 + 0.1 * np.sin(tp * x) * np.cos(tp * y), 1.0 + 0.15 * np.sin(tp * (x + y)))


def _analytic_rhs(x, y, h=1e-4):
    def flux(x, y, axis):
        rho, u, v, p = _smooth_primitives(x, y)
        e = p / (GAMMA - 1.0) + 0.5 * rho * (u * u + v * v)
        vel = u if axis == 0 else v
        return np.stack([rho * vel, rho * u * vel + (p if axis == 0 else 0.0), rho * v * vel + (p if axis == 1 else 0.0),
                         (e + p) * vel], axis=-1)

    def deriv(axis):
        tot = 0.0
        for k, w in ((-2, 1 / 12), (-1, -2 / 3), (1, 2 / 3), (2, -1 / 12)):
            tot = tot + w * flux(x + (k * h if axis == 0 else 0.0), y + (k * h if axis == 1 else 0.0), axis)
        return tot / h

    return -(deriv(0) + deriv(1))


def test_interior_operator_is_fourth_order_accurate():
    from cfd_demo_b200 import rectangle_mesh
    from cfd_demo_b200.euler import primitive_to_conserved

    errors = []
    for n in (8, 16, 32):
        s = make_solver(rectangle_mesh(n, n), fixed_all(FREE_STREAM))
        x, y = s.node_coordinates()
        rhs, _ = s.rhs(primitive_to_conserved(*_smooth_primitives(x, y), GAMMA))
        inside = np.all(s.connectivity.neighbor_element >= 0, axis=1)
        errors.append(float(np.abs(rhs[:, inside] - _analytic_rhs(x, y)[:, inside]).max()))
    assert errors[0] < 5e-2
    orders = [np.log2(a / b) for a, b in zip(errors, errors[1:])]
    assert all(o > 3.5 for o in orders), (errors, orders)


def test_rhs_rejects_a_badly_shaped_state():
    from cfd_demo_b200 import rectangle_mesh

    s = make_solver(rectangle_mesh(2, 2), fixed_all(FREE_STREAM))
    with pytest.raises(ValueError, match="Expected a state of shape"):
        s.rhs(np.zeros((3, 4)))


# ---- limiters and time integration (test_limiting_and_time.py) -----------------------
def smooth_linear_state(s):
    from cfd_demo_b200.euler import primitive_to_conserved

    x, y = s.node_coordinates()
    return primitive_to_conserved(*FREE_STREAM, GAMMA) + np.array([0.05, 0.03, -0.02, 0.07]) * (0.3 * x + 0.2 * y)[..., None]


def test_limiting_preserves_cell_averages():
    s = make_solver(perturbed_mesh(6, 5, seed=5), fixed_all(FREE_STREAM))
    q = smooth_linear_state(s)
    q = q * (1.0 + 0.3 * np.random.default_rng(1).standard_normal(q.shape))
    assert np.abs(s.cell_averages(s.limit(q)) - s.cell_averages(q)).max() < 1e-12


def test_limiter_leaves_a_linear_solution_alone():
    from cfd_demo_b200 import rectangle_mesh

    s = make_solver(rectangle_mesh(8, 8), fixed_all(FREE_STREAM))
    q = smooth_linear_state(s)
    inside = np.all(s.connectivity.neighbor_element >= 0, axis=1)
    assert np.abs(s.limit(q)[:, inside] - q[:, inside]).max() < 1e-12


def test_troubled_cell_limiter_flattens_an_oscillation():
    from cfd_demo_b200 import rectangle_mesh

    s = make_solver(rectangle_mesh(8, 8), fixed_all(FREE_STREAM))
    q = uniform_state(s, FREE_STREAM)
    target = 2 * (4 * 8 + 4)
    R = s.reference
    osc = 0.2 * np.cos(4.0 * np.pi * R.r) * np.cos(3.0 * np.pi * R.s)
    osc -= R.cell_weights @ osc / R.cell_weights.sum()
    q[:, target, 0] += osc
    lim = s.limit(q)
    assert np.abs(lim[:, target] - q[:, target]).max() > 1e-6
    others = np.arange(s.mesh.num_elements) != target
    assert np.abs(lim[:, others] - q[:, others]).max() < 1e-12
    assert np.allclose(R.linear_midpoint_basis @ (R.p1_midpoint @ lim[:, target, 0]), lim[:, target, 0], atol=1e-12)
    assert np.abs(s.cell_averages(lim) - s.cell_averages(q)).max() < 1e-12


def test_unlimited_skips_slope_limiting_but_keeps_positivity():
    from cfd_demo_b200 import rectangle_mesh

    s = make_solver(rectangle_mesh(6, 6), fixed_all(FREE_STREAM), limiter="unlimited")
    q = uniform_state(s, FREE_STREAM)
    q[:, 2 * (3 * 6 + 3), 0] += 0.2 * np.cos(4.0 * np.pi * s.reference.r)
    lim, count = s.limit_with_count(q)
    assert np.abs(lim - q).max() < 1e-13
    assert count == 0


def test_positivity_limiter_repairs_negative_nodes():
    from cfd_demo_b200 import rectangle_mesh
    from cfd_demo_b200.euler import conserved_to_primitive

    s = make_solver(rectangle_mesh(4, 4), fixed_all(FREE_STREAM), limiter="unlimited")
    q = uniform_state(s, (1.0, 0.0, 0.0, 1.0))
    dev = np.linspace(-1.5, 1.5, 15)
    dev -= s.reference.cell_weights @ dev / s.reference.cell_weights.sum()
    q[:, 5, 0] += dev
    q[:, 5, 3] += 1.2 * dev
    assert q[:, 5, 0].min() < 0.0
    lim = s.limit(q)
    rho, _, _, p = conserved_to_primitive(lim, GAMMA)
    assert rho.min() >= 1e-13 * (1.0 - 1e-9)
    assert p.min() >= 1e-13 * (1.0 - 1e-9)
    assert np.abs(s.cell_averages(lim) - s.cell_averages(q)).max() < 1e-12
    untouched = np.arange(s.mesh.num_elements) != 5
    assert np.abs(lim[:, untouched] - q[:, untouched]).max() < 1e-13


def test_time_step_matches_the_cfl_formula():
    from cfd_demo_b200 import rectangle_mesh

    s = make_solver(rectangle_mesh(5, 4), fixed_all(FREE_STREAM))
    q = uniform_state(s, FREE_STREAM)
    rho, u, v, p = FREE_STREAM
    lam = np.hypot(u, v) + np.sqrt(GAMMA * p / rho)
    geo = np.min(2.0 * s.geometry.area[:, None] / (25.0 * s.geometry.edge_length), axis=1)
    assert s.time_step(q) == pytest.approx(0.5 * geo.min() / lam, rel=1e-12)
    finer = make_solver(rectangle_mesh(10, 8), fixed_all(FREE_STREAM))
    assert finer.time_step(uniform_state(finer, FREE_STREAM)) == pytest.approx(0.5 * s.time_step(q), rel=1e-12)


def sod_like_solver(nx=20, ny=2, **cfg):
    from cfd_demo_b200 import EulerSolver, SolverConfig, rectangle_mesh
    from cfd_demo_b200.cases import sod_boundaries

    return EulerSolver(rectangle_mesh(nx, ny), sod_boundaries(),
                       SolverConfig(flux=cfg.pop("flux", "rusanov"), limiter=cfg.pop("limiter", "minmod"), gamma=GAMMA, **cfg))


def initial_sod_state(s):
    from cfd_demo_b200.euler import primitive_to_conserved

    left = primitive_to_conserved(1.0, 0.0, 0.0, 1.0, GAMMA)
    right = primitive_to_conserved(0.125, 0.0, 0.0, 0.1, GAMMA)
    on_left = s.geometry.centroid[:, 0] < 0.5
    q = np.empty(s.state_shape)
    q[:, on_left] = left
    q[:, ~on_left] = right
    return q


def test_ssp_rk3_reaches_the_requested_time_exactly():
    s = sod_like_solver()
    res = s.run(initial_sod_state(s), 0.01)
    assert res.time == pytest.approx(0.01, abs=0.0)
    assert res.steps > 1 and res.rejected_steps == 0 and res.wall_time > 0.0
    assert res.state.shape == s.state_shape


def test_ssp_rk3_is_conservative_over_a_run():
    s = sod_like_solver()
    q = initial_sod_state(s)
    res = s.run(q, 0.01)
    defect = s.integrate(res.state) - s.integrate(q) + res.boundary_flux_integral
    assert np.abs(defect).max() < 1e-13


def test_third_order_convergence_of_the_time_integrator():
    from cfd_demo_b200.euler import primitive_to_conserved

    s = make_solver(perturbed_mesh(5, 4, seed=7), fixed_all(FREE_STREAM), limiter="unlimited")
    x, y = s.node_coordinates()
    q0 = primitive_to_conserved(*FREE_STREAM, GAMMA) * (1.0 + 0.02 * np.sin(2 * np.pi * x) * np.cos(2 * np.pi * y))[..., None]

    def march(q, steps):
        for _ in range(steps):
            q, rep = s.step(q, 0.02 / steps)
            assert rep.admissible
        return q

    ref = march(q0, 64)
    errs = [np.abs(march(q0, n) - ref).max() for n in (4, 8)]
    assert np.log2(errs[0] / errs[1]) > 2.5, errs


def test_run_rejects_an_inadmissible_initial_state():
    from cfd_demo_b200 import SolverError

    s = sod_like_solver()
    q = initial_sod_state(s)
    q[0, 0, 0] = -1.0
    with pytest.raises(SolverError, match="positive nodal density and pressure"):
        s.run(q, 0.01)


def test_run_halves_the_step_and_gives_up_after_max_rejections():
    from cfd_demo_b200 import EulerSolver, SolverConfig, SolverError, rectangle_mesh
    from cfd_demo_b200.cases import sod_boundaries

    s = EulerSolver(rectangle_mesh(4, 2), sod_boundaries(),
                    SolverConfig(flux="rusanov", limiter="minmod", gamma=GAMMA, cfl=1e6, max_rejections=2))
    with pytest.raises(SolverError, match="was rejected 3 times"):
        s.run(initial_sod_state(s), 0.5)


def test_step_reports_stage_minima_and_troubled_cells():
    s = sod_like_solver()
    q = initial_sod_state(s)
    _, rep = s.step(q, s.time_step(q))
    assert rep.min_density > 0.0 and rep.min_pressure > 0.0
    assert rep.troubled_cells > 0 and rep.admissible
    assert rep.boundary_flux.shape == (4,)


# ---- interface fluxes (test_physics.py), on the device flux functions -------------------
def _cons(prim):
    from cfd_demo_b200.euler import primitive_to_conserved

    return primitive_to_conserved(*prim, GAMMA)


def _normal_flux(q, nx, ny):
    from oracle.physics import normal_flux

    return normal_flux(np.asarray(q), nx, ny, GAMMA)


@pytest.mark.parametrize("name", FLUXES)
def test_interface_flux_is_consistent(name):
    from cfd_demo_b200 import get_interface_flux

    f = get_interface_flux(name)
    for prim in STATES:
        q = _cons(prim)
        for nx, ny in ((1.0, 0.0), (0.0, 1.0), (0.6, -0.8)):
            assert np.allclose(f(q, q, nx, ny, GAMMA), _normal_flux(q, nx, ny), atol=1e-12)


@pytest.mark.parametrize("name", FLUXES)
def test_interface_flux_is_conservative(name):
    from cfd_demo_b200 import get_interface_flux

    f = get_interface_flux(name)
    for a in STATES:
        for b in STATES:
            qm, qp = _cons(a), _cons(b)
            for nx, ny in ((1.0, 0.0), (0.6, -0.8)):
                assert np.allclose(f(qm, qp, nx, ny, GAMMA), -f(qp, qm, -nx, -ny, GAMMA), atol=1e-12)


@pytest.mark.parametrize("name", FLUXES)
def test_interface_flux_is_rotationally_invariant(name):
    from cfd_demo_b200 import get_interface_flux

    f = get_interface_flux(name)
    c, s = np.cos(0.7), np.sin(0.7)
    rot = lambda q: np.array([q[0], c * q[1] - s * q[2], s * q[1] + c * q[2], q[3]])  # noqa: E731
    qm, qp = _cons(STATES[2]), _cons(STATES[3])
    nx, ny = 0.6, -0.8
    assert np.allclose(rot(f(qm, qp, nx, ny, GAMMA)), f(rot(qm), rot(qp), c * nx - s * ny, s * nx + c * ny, GAMMA), atol=1e-12)


def test_upwind_fluxes_resolve_a_stationary_contact_exactly():
    from cfd_demo_b200.fluxes import hllc, roe, rusanov

    qm, qp = _cons((1.0, 0.0, 0.0, 1.0)), _cons((0.125, 0.0, 0.0, 1.0))
    exact = _normal_flux(qm, 1.0, 0.0)
    assert np.allclose(roe(qm, qp, 1.0, 0.0, GAMMA), exact, atol=1e-12)
    assert np.allclose(hllc(qm, qp, 1.0, 0.0, GAMMA), exact, atol=1e-12)
    assert not np.allclose(rusanov(qm, qp, 1.0, 0.0, GAMMA), exact, atol=1e-6)


def test_upwind_fluxes_pick_the_supersonic_side():
    from cfd_demo_b200.fluxes import hllc, roe

    r, l = _cons((1.0, 5.0, 0.0, 1.0)), _cons((0.8, 5.0, 0.0, 1.2))
    for f in (roe, hllc):
        assert np.allclose(f(r, l, 1.0, 0.0, GAMMA), _normal_flux(r, 1.0, 0.0), atol=1e-12)
        assert np.allclose(f(l, r, -1.0, 0.0, GAMMA), _normal_flux(r, -1.0, 0.0), atol=1e-12)


def test_rusanov_matches_its_definition():
    from cfd_demo_b200.fluxes import rusanov

    qm, qp = _cons(STATES[2]), _cons(STATES[3])
    nx, ny = 0.6, -0.8
    sp = []
    for q in (qm, qp):
        rho, u, v, p = q[0], q[1] / q[0], q[2] / q[0], 0.4 * (q[3] - 0.5 * (q[1] ** 2 + q[2] ** 2) / q[0])
        sp.append(abs(u * nx + v * ny) + np.sqrt(GAMMA * p / rho))
    exp = 0.5 * (_normal_flux(qm, nx, ny) + _normal_flux(qp, nx, ny) - max(sp) * (qp - qm))
    assert np.allclose(rusanov(qm, qp, nx, ny, GAMMA), exp, atol=1e-14)


def test_hllc_preserves_positivity_for_a_strong_expansion():
    from cfd_demo_b200.fluxes import hllc

    out = hllc(_cons((1.0, -2.0, 0.0, 0.4)), _cons((1.0, 2.0, 0.0, 0.4)), 1.0, 0.0, GAMMA)
    assert np.all(np.isfinite(out)) and out[0] == pytest.approx(0.0, abs=1e-12)


def test_limiter_closed_forms():
    from cfd_demo_b200.limiters import mc, minmod, superbee, van_leer

    r = np.array([-1.0, 0.0, 0.25, 0.5, 1.0, 2.0, 4.0])
    assert np.allclose(minmod(r), [0.0, 0.0, 0.25, 0.5, 1.0, 1.0, 1.0])
    assert np.allclose(mc(r), [0.0, 0.0, 0.5, 0.75, 1.0, 1.5, 2.0])
    assert np.allclose(van_leer(r), [0.0, 0.0, 0.4, 2 / 3, 1.0, 4 / 3, 1.6])
    assert np.allclose(superbee(r), [0.0, 0.0, 0.5, 1.0, 1.0, 2.0, 2.0])


def test_face_pairing_check_on_the_gpu():
    """The setup's coordinate check of the face-node pairing rule, run on the
    device (the path EulerSolver takes), accepts a conforming mesh and rejects
    a wrong neighbour face."""
    import dataclasses

    from cfd_demo_b200 import mesh as pm
    from cfd_demo_b200.operators import check_face_pairing
    from cfd_demo_b200.reference_element import build_reference_triangle

    ref = build_reference_triangle(4)
    m = pm.jittered_rectangle_mesh(40, 30, 0.2, 5)
    conn, geo = pm.build_connectivity(m), pm.element_geometry(m)
    check_face_pairing(m, conn, ref, geometry=geo, device="cuda")
    nf = conn.neighbor_face.copy()
    e, f = np.argwhere(conn.neighbor_element >= 0)[7]
    nf[e, f] = (nf[e, f] + 2) % 3
    with pytest.raises(ValueError, match="not conforming"):
        check_face_pairing(m, dataclasses.replace(conn, neighbor_face=nf), ref, geometry=geo, device="cuda")
