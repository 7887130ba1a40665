"""CPU tests of the host side: reference-element tables (bitwise against the
reference's), mesh/connectivity/geometry against the oracle, the device
table layout, configuration validation, and the C ABI library (loads,
exports every symbol of include/cfd_b200.h, struct layouts agree)."""

from __future__ import annotations

import ctypes as C
import os
import re

import numpy as np
import pytest

import oracle
from tests.golden_io import load

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_tables_are_bitwise_the_references():
    from cfd_demo_b200.reference_element import build_reference_triangle

    g = load("element")
    ref = build_reference_triangle(4)
    for key in ("r", "s", "dr", "ds", "lift", "cell_weights", "face_weights", "p1_midpoint",
                "linear_midpoint_basis", "mass", "vandermonde"):
        assert np.array_equal(getattr(ref, key), g[key]), key
    assert np.array_equal(ref.face_nodes, g["face_nodes"])
    assert np.array_equal(ref.face_midpoint_nodes, g["face_midpoint_nodes"])


def test_generated_tables_header_matches_the_tables():
    from cfd_demo_b200 import build

    path = os.path.join(ROOT, "cfd_demo_b200", "csrc", "tables.cuh")
    assert open(path).read() == build.generate_tables()


@pytest.mark.parametrize("nx,ny,amp,seed", [(1, 1, 0.0, 0), (3, 2, 0.2, 1), (6, 5, 0.25, 0), (9, 4, 0.2, 7)])
def test_mesh_connectivity_geometry_match_oracle(nx, ny, amp, seed):
    from cfd_demo_b200 import mesh as pm

    om = oracle.mesh.perturbed_mesh(nx, ny, amp, seed) if amp else oracle.rectangle_mesh(nx, ny)
    m = pm.TriangleMesh(om.vertices, om.elements, om.boundary_edges)
    c, oc = pm.build_connectivity(m), oracle.build_connectivity(om)
    assert np.array_equal(c.neighbor_element, oc.neighbor_element)
    assert np.array_equal(c.neighbor_face, oc.neighbor_face)
    assert c.boundary_tags == oc.boundary_tags and np.array_equal(c.face_tag, oc.face_tag)
    g, og = pm.element_geometry(m), oracle.element_geometry(om)
    for f in ("jacobian", "rx", "ry", "sx", "sy", "centroid", "normal", "edge_length", "face_midpoint"):
        assert np.array_equal(getattr(g, f), getattr(og, f)), f


def test_rectangle_mesh_matches_oracle_bitwise():
    from cfd_demo_b200.mesh import rectangle_mesh

    for nx, ny, xr, yr in ((4, 3, (0, 1), (0, 1)), (100, 10, (0.0, 1.0), (0.0, 0.1))):
        a, b = rectangle_mesh(nx, ny, xr, yr), oracle.rectangle_mesh(nx, ny, xr, yr)
        assert np.array_equal(a.vertices, b.vertices) and np.array_equal(a.elements, b.elements)
        for t in b.boundary_edges:
            assert np.array_equal(a.boundary_edges[t], b.boundary_edges[t])


def test_face_pairing_rule_matches_coordinate_matching():
    """The kernels pair face node k with node 4-k (or k) of the neighbour's
    face; the reference pairs by coordinates (mesh.py:254-291)."""
    from cfd_demo_b200.mesh import TriangleMesh, build_connectivity
    from cfd_demo_b200.reference_element import build_reference_triangle

    om = oracle.mesh.perturbed_mesh(7, 5, 0.25, 3)
    ref = build_reference_triangle()
    conn = oracle.build_connectivity(om)
    x, y = oracle.node_coordinates(om, ref.r, ref.s)
    partner = oracle.pair_face_nodes(om, conn, x, y, ref.face_nodes)
    fn = ref.face_nodes
    for f in range(3):
        el = np.flatnonzero(conn.neighbor_element[:, f] >= 0)
        nf = conn.neighbor_face[el, f]
        same = (f == 2) != (nf == 2)
        for k in range(5):
            expect = fn[nf, np.where(same, k, 4 - k)]
            assert np.array_equal(partner[f, k, el], expect)
    from cfd_demo_b200.operators import check_face_pairing

    check_face_pairing(TriangleMesh(om.vertices, om.elements, om.boundary_edges),
                       build_connectivity(TriangleMesh(om.vertices, om.elements, om.boundary_edges)), ref)


def test_cockburn_shu_coefficients_match_oracle():
    from cfd_demo_b200 import mesh as pm
    from cfd_demo_b200.operators import neighbor_coefficients
    from oracle.physics import FixedState, SlipWall

    om = oracle.mesh.perturbed_mesh(6, 4, 0.2, 2)
    fs = FixedState((1.0, 0.1, 0.0, 2.5))
    s = oracle.OracleSolver(om, {"left": fs, "right": fs, "bottom": SlipWall(), "top": SlipWall()},
                            flux="rusanov", limiter="minmod", gamma=1.4)
    m = pm.TriangleMesh(om.vertices, om.elements, om.boundary_edges)
    a, b, p = neighbor_coefficients(pm.build_connectivity(m), pm.element_geometry(m))
    assert np.array_equal(a.T, s.alpha) and np.array_equal(b.T, s.beta) and np.array_equal(p.T, s.partner_face)


def test_limiter_operators_match_oracle_tables():
    """EulerSolver.limiter_operators (the reference's LimiterOperators fields)
    against the oracle's limiter tables."""
    from cfd_demo_b200 import mesh as pm
    from cfd_demo_b200.boundary import FixedState as PFixed, SlipWall as PSlip
    from cfd_demo_b200.operators import limiter_operators, resolve_boundary_conditions
    from cfd_demo_b200.reference_element import build_reference_triangle
    from oracle.physics import FixedState, SlipWall

    om = oracle.mesh.perturbed_mesh(6, 4, 0.2, 2)
    st = (1.0, 0.1, 0.0, 2.5)
    s = oracle.OracleSolver(om, {"left": FixedState(st), "right": FixedState(st), "bottom": SlipWall(),
                                 "top": SlipWall()}, flux="rusanov", limiter="minmod", gamma=1.4)
    m = pm.TriangleMesh(om.vertices, om.elements, om.boundary_edges)
    conn, geo = pm.build_connectivity(m), pm.element_geometry(m)
    kind, state = resolve_boundary_conditions(conn, {"left": PFixed(st), "right": PFixed(st), "bottom": PSlip(),
                                                     "top": PSlip()})
    lo = limiter_operators(conn, geo, build_reference_triangle(4), kind, state)
    assert np.array_equal(lo.average_weights, s.avg_weights)
    assert np.array_equal(lo.neighbor, s.nbr3) and np.array_equal(lo.neighbor_kind, s.kind3)
    assert np.array_equal(lo.normal_x, s.nx3) and np.array_equal(lo.normal_y, s.ny3)
    assert np.array_equal(lo.fixed_state, s.fixed3)
    assert np.array_equal(lo.alpha, s.alpha) and np.array_equal(lo.beta, s.beta)
    assert np.array_equal(lo.partner_face, s.partner_face)
    assert lo.p1_midpoint.shape == (3, 15) and lo.linear_basis.shape == (15, 3) and lo.midpoint_nodes.shape == (3,)


def test_host_tables_layout():
    from cfd_demo_b200 import FixedState, SlipWall
    from cfd_demo_b200 import mesh as pm
    from cfd_demo_b200.operators import host_tables, resolve_boundary_conditions
    from cfd_demo_b200.reference_element import build_reference_triangle

    m = pm.rectangle_mesh(5, 3)
    conn, geo = pm.build_connectivity(m), pm.element_geometry(m)
    bcs = {"left": FixedState((1, 0, 0, 2.5)), "right": FixedState((0.125, 0, 0, 0.25)), "bottom": SlipWall(), "top": SlipWall()}
    kind, state = resolve_boundary_conditions(conn, bcs)
    h = host_tables(m, conn, geo, build_reference_triangle(), kind, state)
    for f in range(3):
        k = (h.face_info >> (8 * f)) & 3
        assert np.array_equal(k, kind[:, f])
        interior = k == 0
        assert np.array_equal(h.neighbor[f][interior], conn.neighbor_element[interior, f])
        assert np.array_equal((h.face_info >> (8 * f + 2))[interior] & 3, conn.neighbor_face[interior, f])
        fixed = k == 2
        assert np.array_equal(h.bc_states[h.neighbor[f][fixed]], state[fixed, f])
    assert np.allclose(h.face_geo[2], 0.5 * geo.edge_length[:, 0] / geo.jacobian)


def test_boundary_condition_errors_match_reference():
    from cfd_demo_b200 import FixedState, SlipWall
    from cfd_demo_b200 import mesh as pm
    from cfd_demo_b200.operators import resolve_boundary_conditions

    conn = pm.build_connectivity(pm.rectangle_mesh(2, 2))
    with pytest.raises(ValueError, match="Boundary tags without a boundary condition"):
        resolve_boundary_conditions(conn, {"left": SlipWall()})
    with pytest.raises(ValueError, match="not in the mesh"):
        resolve_boundary_conditions(conn, {t: SlipWall() for t in ("left", "right", "top", "bottom", "front")})
    with pytest.raises(ValueError, match="four finite"):
        FixedState((1.0, 0.0, np.nan, 1.0))


def test_mesh_validation_errors():
    from cfd_demo_b200 import mesh as pm

    m = pm.rectangle_mesh(2, 1)
    with pytest.raises(ValueError, match="counterclockwise"):
        pm.TriangleMesh(m.vertices, m.elements[:, ::-1], m.boundary_edges)
    bad = dict(m.boundary_edges)
    bad.pop("top")
    with pytest.raises(ValueError, match="has no tag"):
        pm.build_connectivity(pm.TriangleMesh(m.vertices, m.elements, bad))
    with pytest.raises(ValueError, match="nx and ny must be positive"):
        pm.rectangle_mesh(0, 3)


def test_solver_config_validates_its_options():
    from cfd_demo_b200 import SolverConfig

    with pytest.raises(ValueError, match="Unknown interface flux"):
        SolverConfig(flux="godunov", limiter="minmod", gamma=1.4)
    with pytest.raises(ValueError, match="Unknown limiter"):
        SolverConfig(flux="rusanov", limiter="ospre", gamma=1.4)
    with pytest.raises(ValueError, match="gamma"):
        SolverConfig(flux="rusanov", limiter="minmod", gamma=1.0)
    with pytest.raises(ValueError, match="cfl"):
        SolverConfig(flux="rusanov", limiter="minmod", gamma=1.4, cfl=0.0)
    with pytest.raises(ValueError, match="precision"):
        SolverConfig(flux="rusanov", limiter="minmod", gamma=1.4, precision="fp16")


def test_library_exports_every_declared_symbol():
    from cfd_demo_b200 import _native

    lib = _native.load()
    header = open(os.path.join(ROOT, "include", "cfd_b200.h")).read()
    declared = sorted(set(re.findall(r"^\s*(?:int|int64_t|const char\*)\s+(cfd_\w+)\s*\(", header, re.M)))
    assert declared, "no declarations found"
    for name in declared:
        assert hasattr(lib, name), name
    assert set(declared) <= set(_native.exported_symbols()) | {"cfd_struct_sizes"}
    assert lib.cfd_abi_version() == _native.ABI_VERSION
    assert f"#define CFD_ABI_VERSION {_native.ABI_VERSION}" in header


def test_struct_layouts_agree_with_the_header():
    from cfd_demo_b200 import _native

    lib = _native.load()
    out = (C.c_int32 * 5)()
    assert lib.cfd_struct_sizes(out, 5) == 0
    names = ["CfdMesh", "CfdStageAcc", "CfdStepReport", "CfdControl", "CfdSolver"]
    assert list(out) == [_native.SIZES[n] for n in names]


def test_argument_errors_are_reported_without_a_gpu():
    from cfd_demo_b200 import _native

    lib = _native.load()
    assert lib.cfd_rhs(None, None, None, None, None) == -1
    assert b"null solver" in lib.cfd_last_error()
    assert lib.cfd_interface_flux(7, 1, 1, 1, 1, 1, 1.4, 1, None) == -1
    assert lib.cfd_limiter_phi(0, -1, None, None, None) == -1
    assert lib.cfd_rk3_step_fixed(None, None, None, None, None, None, None) == -1
    assert lib.cfd_rk3_step_adjoint(None, None, None, None, None, None, None, 0, None, None) == -1


def test_adjoint_buffer_sizes():
    from cfd_demo_b200 import _native

    lib = _native.load()
    ld = 128
    # tape: five stage states (before / after limiting) + 3 x (4 averages + 3 minima / wave speed
    # + 2 positivity theta / node) doubles
    assert lib.cfd_tape_bytes(ld, _native.CFD_FP64) == 5 * 60 * ld * 8 + 27 * ld * 8
    assert lib.cfd_tape_bytes(ld, _native.CFD_FP32_MIXED) == 5 * 60 * ld * 4 + 27 * ld * 8
    # adjoint scratch: 252 rows of reals, the replay list (ld ints), its counter slot, the listed
    # flags (ld bytes rounded up to 256)
    assert lib.cfd_adjoint_work_bytes(ld, _native.CFD_FP64) == 252 * ld * 8 + 4 * ld + 256 + 256
    assert lib.cfd_adjoint_work_bytes(300, _native.CFD_FP32_MIXED) == 252 * 300 * 4 + 4 * 300 + 256 + 512
    assert lib.cfd_tape_bytes(0, _native.CFD_FP64) == -1
    assert lib.cfd_adjoint_work_bytes(ld, 9) == -1


def test_package_has_no_oracle_dependency():
    """The product never imports the oracle (it is the checker)."""
    pkg = os.path.join(ROOT, "cfd_demo_b200")
    for dirpath, _, files in os.walk(pkg):
        for f in files:
            if f.endswith(".py"):
                text = open(os.path.join(dirpath, f)).read()
                assert "import oracle" not in text and "from oracle" not in text, f


def test_face_pairing_check_rejects_a_wrong_neighbour_face():
    import dataclasses

    from cfd_demo_b200 import mesh as pm
    from cfd_demo_b200.operators import check_face_pairing
    from cfd_demo_b200.reference_element import build_reference_triangle

    ref = build_reference_triangle(4)
    m = pm.jittered_rectangle_mesh(6, 5, 0.2, 1)
    conn, geo = pm.build_connectivity(m), pm.element_geometry(m)
    check_face_pairing(m, conn, ref, geometry=geo)
    nf = conn.neighbor_face.copy()
    e, f = np.argwhere(conn.neighbor_element >= 0)[0]
    nf[e, f] = (nf[e, f] + 1) % 3
    with pytest.raises(ValueError, match="not conforming"):
        check_face_pairing(m, dataclasses.replace(conn, neighbor_face=nf), ref, geometry=geo)
