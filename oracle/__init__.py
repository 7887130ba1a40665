"""CPU oracle for the CFD-demo DG hot path — TEST INFRASTRUCTURE ONLY.

This package restates, in plain NumPy float64 and in the reference's own
array layout (node, element, variable) = (Np, K, 4), the algorithm of
CFD-demo's solver: the degree-4 nodal reference triangle, the rectangle mesh
and its connectivity, the collocated strong-form DG right-hand side with the
Rusanov / Roe / HLLC interface fluxes, the Cockburn-Shu troubled-cell limiter
with its five phi(r) functions, the Zhang-Shu positivity limiter, the SSP-RK3
step with its report, the CFL time step and the host run loop. Every function
cites the reference file:line it follows (paths relative to the CFD-demo
project root).

It is the checker, never the product: only ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline arm of ``bench.py`` may
import it. The shipped package (``cfd_demo_b200``) never imports it and has no
CPU fallback.

Parity of this restatement is pinned against golden vectors generated by the
reference's own source (``tests/golden/make_golden.py``), checked in
``tests/test_oracle_golden.py``.
"""

from .element import ReferenceTriangle, build_reference_triangle
from .mesh import (
    ElementGeometry,
    MeshConnectivity,
    TriangleMesh,
    build_connectivity,
    element_geometry,
    node_coordinates,
    pair_face_nodes,
    rectangle_mesh,
)
from .physics import (
    EXACT_STATE,
    FIXED_STATE,
    SLIP_WALL,
    ExactState,
    FixedState,
    SlipWall,
    cartesian_fluxes,
    conserved_to_primitive,
    get_interface_flux,
    get_limiter_function,
    normal_flux,
    pressure,
    primitive_to_conserved,
    sound_speed,
)
from .solver import OracleSolver, RunResult, SolverError, StepReport, sod_shock_tube

__all__ = [
    "EXACT_STATE",
    "ExactState",
    "FIXED_STATE",
    "SLIP_WALL",
    "ElementGeometry",
    "FixedState",
    "MeshConnectivity",
    "OracleSolver",
    "ReferenceTriangle",
    "RunResult",
    "SlipWall",
    "SolverError",
    "StepReport",
    "TriangleMesh",
    "build_connectivity",
    "build_reference_triangle",
    "cartesian_fluxes",
    "conserved_to_primitive",
    "element_geometry",
    "get_interface_flux",
    "get_limiter_function",
    "node_coordinates",
    "normal_flux",
    "pair_face_nodes",
    "pressure",
    "primitive_to_conserved",
    "rectangle_mesh",
    "sod_shock_tube",
    "sound_speed",
]
