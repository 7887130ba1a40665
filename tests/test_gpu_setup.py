"""The mesh tables built on the GPU (cfd_mesh_build) against the host builder:
geometry (mesh.py:216-243 of CFD-demo), connectivity and boundary tags
(mesh.py:135-185), Cockburn-Shu coefficients (limiting.py:51-94) and the
packed neighbour / face-info rows must be equal bit for bit, on rectangles,
jittered meshes, the golden fixtures' meshes and the 1M-triangle benchmark
mesh; invalid meshes must fail with the host builder's errors."""

from __future__ import annotations

import time

import numpy as np
import pytest

from tests.golden_io import GAMMA, boundary_specs, case_prefixes, load, mesh_parts

pytestmark = pytest.mark.gpu

FIELDS = ("metric", "face_geo", "face_hlen", "dt_geo", "jacobian", "cs_coef", "neighbor", "face_info", "bc_states")


def _host_and_device(mesh, bcs):
    from cfd_demo_b200 import _native
    from cfd_demo_b200.mesh import build_connectivity, element_geometry
    from cfd_demo_b200.operators import DeviceTables, host_tables, resolve_boundary_conditions
    from cfd_demo_b200.reference_element import build_reference_triangle

    ref = build_reference_triangle(4)
    conn = build_connectivity(mesh)
    geo = element_geometry(mesh)
    kind, state = resolve_boundary_conditions(conn, bcs)
    host = DeviceTables([host_tables(mesh, conn, geo, ref, kind, state)], "cuda", _native.CFD_FP64)
    dev = DeviceTables.build_on_device(mesh, bcs, ref, "cuda", _native.CFD_FP64)
    return host, dev


def _assert_same(host, dev):
    assert (host.num_elements, host.ld) == (dev.num_elements, dev.ld)
    for name in FIELDS:
        a, b = getattr(host, name), getattr(dev, name)
        assert a.shape == b.shape, name
        assert a.dtype == b.dtype, name
        # padding columns beyond K are zero in both
        assert bool((a == b).all()), (name, int((a != b).sum()))


def _sod_bcs():
    from cfd_demo_b200.cases import sod_boundaries

    return sod_boundaries()


@pytest.mark.parametrize("nx,ny,amp,seed", [(1, 1, 0.0, 0), (3, 2, 0.0, 0), (9, 4, 0.2, 7), (40, 33, 0.25, 3),
                                            (100, 10, 0.0, 0)])
def test_device_tables_equal_the_host_tables(nx, ny, amp, seed):
    from cfd_demo_b200 import FixedState, SlipWall, jittered_rectangle_mesh, rectangle_mesh

    mesh = rectangle_mesh(nx, ny) if amp == 0.0 else jittered_rectangle_mesh(nx, ny, amp, seed)
    walls = {t: SlipWall() for t in ("left", "right", "bottom", "top")}
    fixed = {"left": FixedState.from_primitive(1.0, 0.1, 0.0, 1.0, GAMMA),
             "right": FixedState.from_primitive(0.5, 0.0, 0.2, 0.4, GAMMA),
             "bottom": SlipWall(), "top": FixedState.from_primitive(1.0, 0.1, 0.0, 1.0, GAMMA)}
    for bcs in (walls, fixed):
        _assert_same(*_host_and_device(mesh, bcs))


@pytest.mark.parametrize("fixture", ["rhs", "limit", "step"])
def test_device_tables_of_the_golden_meshes(fixture):
    from cfd_demo_b200 import FixedState, SlipWall, TriangleMesh

    g = load(fixture)
    for prefix in case_prefixes(g):
        v, e, edges = mesh_parts(g, prefix)
        bcs = {t: (SlipWall() if k == 1 else FixedState(s)) for t, (k, s) in boundary_specs(g, prefix).items()}
        _assert_same(*_host_and_device(TriangleMesh(v, e, edges), bcs))


def test_device_tables_of_the_benchmark_mesh(report):
    """The 1M-triangle benchmark mesh: equal tables, and the setup time of
    the solver (GPU tables) against the host builder's."""
    import torch

    from cfd_demo_b200 import EulerSolver, SolverConfig
    from cfd_demo_b200.workloads import microbenchmark_boundaries, microbenchmark_mesh

    mesh = microbenchmark_mesh()
    bcs = microbenchmark_boundaries()
    host, dev = _host_and_device(mesh, bcs)
    _assert_same(host, dev)
    cfg = SolverConfig(flux="roe", limiter="unlimited", gamma=GAMMA)
    EulerSolver(mesh, bcs, cfg)  # warm: library, context
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    EulerSolver(mesh, bcs, cfg)
    torch.cuda.synchronize()
    gpu_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    _host_and_device(mesh, bcs)
    host_s = time.perf_counter() - t0
    report(f"1M-triangle mesh setup: EulerSolver with GPU-built tables {gpu_s:.2f} s; host builder + upload "
           f"(+ GPU build for the comparison) {host_s:.2f} s")
    assert gpu_s < 2.0


def _bad(mesh_fn):
    from cfd_demo_b200 import EulerSolver, SlipWall, SolverConfig

    mesh = mesh_fn()
    bcs = {t: SlipWall() for t in mesh.boundary_edges}
    with pytest.raises(ValueError) as dev_err:
        EulerSolver(mesh, bcs, SolverConfig(flux="rusanov", limiter="minmod", gamma=GAMMA))
    return str(dev_err.value)


def test_invalid_meshes_fail_with_the_host_builders_errors():
    from cfd_demo_b200 import TriangleMesh, rectangle_mesh
    from cfd_demo_b200.mesh import build_connectivity

    base = rectangle_mesh(3, 2)

    def untagged():
        edges = dict(base.boundary_edges)
        edges["top"] = edges["top"][1:]
        return TriangleMesh(base.vertices, base.elements, edges)

    def doubly_tagged():
        edges = dict(base.boundary_edges)
        edges["extra"] = edges["left"][:1]
        return TriangleMesh(base.vertices, base.elements, edges)

    def interior_tagged():
        edges = dict(base.boundary_edges)
        edges["extra"] = np.array([[0, 5]])  # the diagonal of cell (0, 0)
        return TriangleMesh(base.vertices, base.elements, edges)

    def nonconforming():  # a third element on the diagonal of cell (0, 0)
        v = np.vstack([base.vertices, [[0.1, 0.4]]])
        e = np.vstack([base.elements, [[0, 5, len(v) - 1]]])
        return TriangleMesh(v, e, base.boundary_edges)

    for make in (untagged, doubly_tagged, interior_tagged, nonconforming):
        with pytest.raises(ValueError) as host_err:
            build_connectivity(make())
        assert _bad(make) == str(host_err.value), make.__name__
