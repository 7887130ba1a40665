"""Host side of the oblique-shock case (CFD-demo's proposed ADR 0011 / 0012,
not implemented in the reference): the exact theta-beta-M solution, the
sheared rectangle mesh, the exact-state boundary rows of the device tables,
and the oracle's restatement of the exact-state boundary (CPU only)."""

from __future__ import annotations

import math

import numpy as np
import pytest

GAMMA = 1.4


def _exact(mach=2.0, deg=10.0):
    from cfd_demo_b200.verification import ObliqueShock

    return ObliqueShock(mach, math.radians(deg), GAMMA)


def test_theta_beta_mach_textbook_values():
    """Published oblique-shock values for M1 = 2, theta = 10 deg (weak shock):
    beta = 39.31 deg, p2/p1 = 1.707, rho2/rho1 = 1.458, M2 = 1.641;
    theta_max(M1 = 2) = 22.97 deg; M1 = 3, theta = 15 deg: beta = 32.24 deg."""
    o = _exact()
    assert math.degrees(o.beta) == pytest.approx(39.314, abs=1e-3)
    assert o.downstream[3] / o.upstream[3] == pytest.approx(1.7066, abs=1e-4)
    assert o.downstream[0] == pytest.approx(1.4584, abs=1e-4)
    assert o.downstream_mach == pytest.approx(1.6405, abs=1e-4)
    assert math.degrees(o.theta_max) == pytest.approx(22.9735, abs=1e-4)
    assert math.degrees(_exact(3.0, 15.0).beta) == pytest.approx(32.240, abs=1e-3)


@pytest.mark.parametrize("mach", [1.5, 2.0, 3.0, 5.0])
def test_theta_beta_round_trip_and_limits(mach):
    from cfd_demo_b200.verification import ObliqueShock

    theta_max, beta_max = ObliqueShock.max_deflection(mach, GAMMA)
    for frac in (0.01, 0.3, 0.7, 0.999):
        o = ObliqueShock(mach, frac * theta_max, GAMMA)
        assert ObliqueShock.deflection(mach, o.beta, GAMMA) == pytest.approx(frac * theta_max, rel=1e-12)
        assert math.asin(1.0 / mach) < o.beta < beta_max
        # the post-shock flow is parallel to the wall
        assert math.atan2(o.downstream[2], o.downstream[1]) == pytest.approx(frac * theta_max, rel=1e-12)
    # theta -> 0: beta -> the Mach angle; theta -> theta_max: beta -> beta_max
    assert ObliqueShock(mach, 1e-9, GAMMA).beta == pytest.approx(math.asin(1.0 / mach), abs=1e-6)
    assert ObliqueShock(mach, theta_max * (1 - 1e-10), GAMMA).beta == pytest.approx(beta_max, abs=1e-3)


def test_normal_shock_jumps_conserve_fluxes():
    """Mass, normal momentum, tangential velocity and total enthalpy across
    the shock line."""
    o = _exact(2.5, 12.0)
    n = np.array([math.sin(o.beta), -math.cos(o.beta)])
    t = np.array([math.cos(o.beta), math.sin(o.beta)])
    g = GAMMA

    def fluxes(prim):
        rho, u, v, p = prim
        vel = np.array([u, v])
        un, ut = vel @ n, vel @ t
        h = g / (g - 1) * p / rho + 0.5 * (u * u + v * v)
        return np.array([rho * un, rho * un * un + p, ut, h])

    np.testing.assert_allclose(fluxes(o.upstream), fluxes(o.downstream), rtol=1e-12)


def test_invalid_oblique_inputs():
    from cfd_demo_b200.verification import ObliqueShock

    with pytest.raises(ValueError):
        ObliqueShock(1.0, 0.1)
    with pytest.raises(ValueError):
        ObliqueShock(2.0, 0.0)
    with pytest.raises(ValueError):
        ObliqueShock(2.0, math.radians(23.0))  # above theta_max(2) = 22.97 deg


def test_sheared_mesh():
    from cfd_demo_b200.mesh import build_connectivity, rectangle_mesh, sheared_rectangle_mesh, signed_areas

    flat = rectangle_mesh(6, 4, (0.0, 1.0), (0.0, 0.5))
    zero = sheared_rectangle_mesh(6, 4, 0.0, (0.0, 1.0), (0.0, 0.5))
    assert np.array_equal(zero.vertices, flat.vertices) and np.array_equal(zero.elements, flat.elements)
    th = math.radians(10.0)
    m = sheared_rectangle_mesh(6, 4, th, (0.0, 1.0), (0.0, 0.5))
    assert m.num_elements == 48 and np.array_equal(m.elements, flat.elements)
    assert np.all(signed_areas(m) > 0)
    for tag in ("left", "right", "bottom", "top"):
        assert np.array_equal(m.boundary_edges[tag], flat.boundary_edges[tag])
    # bottom is the inclined wall y = x tan(theta)
    b = m.vertices[np.unique(m.boundary_edges["bottom"])]
    np.testing.assert_allclose(b[:, 1], b[:, 0] * math.tan(th), atol=1e-15)
    conn = build_connectivity(m)
    assert int((conn.neighbor_element < 0).sum()) == 2 * (6 + 4)
    with pytest.raises(ValueError):
        sheared_rectangle_mesh(2, 2, 0.5 * math.pi)


def test_exact_cell_average_matches_sampling():
    from cfd_demo_b200.boundary import ExactState
    from cfd_demo_b200.operators import sampled_cell_average

    o = _exact()
    rng = np.random.default_rng(0)
    tri = rng.uniform(0.0, 1.0, size=(40, 3, 2))
    exact = o.cell_average(tri)
    sampled = sampled_cell_average(ExactState(o.conserved), tri, subdivisions=128)
    jump = np.abs(np.array(o._conserved(o.downstream)) - np.array(o._conserved(o.upstream)))
    assert np.all(np.abs(exact - sampled) <= 0.02 * jump + 1e-12)
    # a triangle wholly on one side averages to that side's state
    far = np.array([[[0.5, 0.9], [0.6, 0.9], [0.5, 1.0]]])
    np.testing.assert_allclose(o.cell_average(far)[0], o._conserved(o.upstream), rtol=1e-15)


def _host_case(nx=8, ny=4):
    from cfd_demo_b200.boundary import ExactState, FixedState, SlipWall
    from cfd_demo_b200.mesh import build_connectivity, element_geometry, sheared_rectangle_mesh
    from cfd_demo_b200.operators import host_tables, resolve_boundary_conditions
    from cfd_demo_b200.reference_element import build_reference_triangle

    o = _exact()
    mesh = sheared_rectangle_mesh(nx, ny, o.theta, (0.0, 1.0), (0.0, 0.5))
    far = ExactState(o.conserved, cell_average=o.cell_average)
    bcs = {"left": FixedState.from_primitive(*o.upstream, gamma=GAMMA), "bottom": SlipWall(), "top": far,
           "right": far}
    ref = build_reference_triangle(4)
    conn = build_connectivity(mesh)
    geo = element_geometry(mesh)
    kind, state = resolve_boundary_conditions(conn, bcs)
    return o, mesh, bcs, ref, conn, host_tables(mesh, conn, geo, ref, kind, state, boundary_conditions=bcs), kind


def test_exact_state_rows_of_the_host_tables():
    """Each exact-state face points at 6 bc_states rows: the function at its
    5 face nodes (element face-node order) and the reflected element's exact
    average."""
    from cfd_demo_b200.mesh import node_coordinates
    from cfd_demo_b200.operators import reflected_triangles

    o, mesh, _, ref, conn, t, kind = _host_case()
    x, y = node_coordinates(mesh, ref.r, ref.s)
    es, fs = np.nonzero(kind == 3)
    assert len(es) == 8 + 4  # top + right faces
    info = t.face_info
    for e, f in zip(es, fs):
        assert (info[e] >> (8 * f)) & 3 == 3
        row = t.neighbor[f, e]
        nodes = ref.face_nodes[f]
        np.testing.assert_array_equal(t.bc_states[row:row + 5], o.conserved(x[nodes, e], y[nodes, e]))
        np.testing.assert_array_equal(t.bc_states[row + 5], o.cell_average(reflected_triangles(mesh, np.array([e]),
                                                                                                np.array([f])))[0])
    # the fixed-state rows come first
    assert t.neighbor[:, :][(np.stack([(info >> (8 * f)) & 3 for f in range(3)]) == 2)].max() == 0


def test_without_the_boundary_conditions_exact_faces_are_refused():
    from cfd_demo_b200.mesh import element_geometry
    from cfd_demo_b200.operators import host_tables, resolve_boundary_conditions

    o, mesh, bcs, ref, conn, _, _ = _host_case()
    kind, state = resolve_boundary_conditions(conn, bcs)
    with pytest.raises(ValueError, match="Exact-state faces"):
        host_tables(mesh, conn, element_geometry(mesh), ref, kind, state)


def test_oracle_oblique_case_conserves_and_matches_the_host_rows():
    """The oracle's exact-state exterior states and ghost averages are the
    host tables' rows; 20 oracle steps conserve mass, momentum and energy to
    round-off against the time-integrated boundary fluxes."""
    import oracle
    from oracle.physics import ExactState as OExact, FixedState as OFixed, SlipWall as OSlip

    o, mesh, _, ref, conn, t, kind = _host_case()
    om = oracle.mesh.TriangleMesh(np.array(mesh.vertices), np.array(mesh.elements),
                                  {k: np.array(v) for k, v in mesh.boundary_edges.items()})
    far = OExact(o.conserved, o.cell_average)
    s = oracle.OracleSolver(om, {"left": OFixed.from_primitive(*o.upstream, GAMMA), "bottom": OSlip(), "top": far,
                                 "right": far}, flux="rusanov", limiter="minmod", gamma=GAMMA)
    es, fs = np.nonzero(kind == 3)
    for e, f in zip(es, fs):
        row = t.neighbor[f, e]
        np.testing.assert_array_equal(s.fixed3[f, e], t.bc_states[row + 5])
        np.testing.assert_array_equal(s.state_fn[f * 5:(f + 1) * 5, e], t.bc_states[row:row + 5])
    q = np.broadcast_to(np.array(OFixed.from_primitive(*o.upstream, GAMMA).state), s.state_shape).copy()
    i0, bf = s.integrate(q), np.zeros(4)
    for _ in range(20):
        q, rep = s.step(q, s.time_step(q))
        assert rep.admissible
        bf += rep.boundary_flux
    assert np.abs(s.integrate(q) - i0 + bf).max() < 1e-12
