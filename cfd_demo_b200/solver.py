"""EulerSolver on one B200: the drop-in for CFD-demo's src/cfd_demo/solver.py.

Same construction (mesh, boundary conditions, SolverConfig), same methods
(rhs, limit, time_step, step, cell_averages, integrate, run), same results and
errors; the numerics run in the sm_100a kernels of libcfd_b200.so. Inputs are
array-likes of shape (Np, K, 4) coerced to float64 (or CUDA tensors of that
shape); outputs are NumPy arrays, as in the reference.

``run`` keeps the reference's loop semantics exactly (CFL dt, shortened last
step, reject-and-halve up to max_rejections, RK-weighted boundary-flux
accumulation, minima, troubled-cell maximum) but executes the loop body on
the device (cfd_run_control), so the host only polls the loop state once per
chunk of attempts, and each chunk is replayed from a CUDA graph.
"""

from __future__ import annotations

import ctypes as C
import time
from collections.abc import Mapping
from dataclasses import dataclass
from types import MappingProxyType
from typing import NamedTuple

import numpy as np

from . import _native
from .boundary import EXACT_STATE, BoundaryCondition
from .euler import NUM_VARIABLES
from .fluxes import FLUX_IDS, get_interface_flux
from .limiters import LIMITER_IDS, get_limiter_function
from .mesh import TriangleMesh, build_connectivity, element_geometry, node_coordinates
from .operators import (DeviceTables, LimiterOperators, exact_state_rows, limiter_operators,
                        resolve_boundary_conditions)
from .reference_element import DEGREE, build_reference_triangle

DEFAULT_CFL = 0.5  # time_integration.py:18
MAX_REJECTIONS = 10  # time_integration.py:19
PRECISIONS = {"fp64": _native.CFD_FP64, "fp32_mixed": _native.CFD_FP32_MIXED}


class SolverError(RuntimeError):
    """Raised when the solver cannot advance an admissible solution."""


@dataclass(frozen=True)
class SolverConfig:
    """Solver configuration (solver.py:37-59), plus the arithmetic form:
    ``precision`` "fp64" (the plain method) or "fp32_mixed"."""

    flux: str
    limiter: str
    gamma: float
    cfl: float = DEFAULT_CFL
    max_rejections: int = MAX_REJECTIONS
    precision: str = "fp64"

    def __post_init__(self) -> None:
        get_interface_flux(self.flux)
        get_limiter_function(self.limiter)
        if not self.gamma > 1.0:
            raise ValueError("gamma must be greater than one.")
        if not self.cfl > 0.0:
            raise ValueError("cfl must be positive.")
        if self.max_rejections < 0:
            raise ValueError("max_rejections must be nonnegative.")
        if self.precision not in PRECISIONS:
            raise ValueError(f"Unknown precision {self.precision!r}; choose one of: {', '.join(PRECISIONS)}.")


class StepReport(NamedTuple):
    """Diagnostics of one SSP-RK3 step (time_integration.py:22-29)."""

    boundary_flux: np.ndarray
    admissible: bool
    min_density: float
    min_pressure: float
    troubled_cells: int


@dataclass(frozen=True, eq=False)
class RunResult:
    """Outcome of EulerSolver.run (solver.py:62-88)."""

    state: np.ndarray
    time: float
    steps: int
    rejected_steps: int
    boundary_flux_integral: np.ndarray
    min_density: float
    min_pressure: float
    max_troubled_cells: int
    wall_time: float


def _stream():
    import torch

    return torch.cuda.current_stream().cuda_stream


class Workspace:
    """Caller-owned device buffers of one solver (states and scratch)."""

    def __init__(self, ops: DeviceTables, precision: int, limited: bool):
        import torch

        dev = ops.device
        n = ops.num_instances
        dtype = torch.float64 if precision == _native.CFD_FP64 else torch.float32
        self.dtype = dtype
        shape = (NUM_VARIABLES * 15, ops.ld)
        self.x0 = torch.zeros(shape, dtype=dtype, device=dev)
        self.x1 = torch.zeros(shape, dtype=dtype, device=dev)
        self.stage = torch.zeros(shape, dtype=dtype, device=dev)
        self.out = torch.zeros(shape, dtype=dtype, device=dev)
        self.averages = torch.zeros((4, ops.ld), dtype=torch.float64, device=dev)
        self.aux = torch.zeros((3, ops.ld), dtype=torch.float64, device=dev)
        self.acc = torch.zeros(3 * n * _native.SIZES["CfdStageAcc"], dtype=torch.uint8, device=dev)
        self.report = torch.zeros(n * _native.SIZES["CfdStepReport"], dtype=torch.uint8, device=dev)
        self.control = torch.zeros(n * _native.SIZES["CfdControl"], dtype=torch.uint8, device=dev)
        self.small = torch.zeros(max(4 * n, 3 * n, 8), dtype=torch.float64, device=dev)
        self.small_i = torch.zeros(max(n, 8), dtype=torch.int32, device=dev)
        # the two-pass limiter's counters and element list
        self.limit_list = torch.zeros(_native.LIMIT_LIST_HEADER + ops.ld, dtype=torch.int32, device=dev)
        # per-stage troubled-cell indicator, written only when recording is on
        self.flags = torch.zeros((3, ops.ld), dtype=torch.uint8, device=dev)


class EulerSolver:
    """Degree-four nodal DG solver for the 2D Euler equations on a B200."""

    def __init__(self, mesh: TriangleMesh, boundary_conditions: Mapping[str, BoundaryCondition], config: SolverConfig,
                 *, device="cuda", block_size: int = 0, graph_chunk: int = 32, variant: int = 0) -> None:
        import torch

        if not torch.cuda.is_available():
            raise RuntimeError("cfd_demo_b200 needs a CUDA GPU (B200); there is no CPU fallback.")
        self.mesh = mesh
        self.config = config
        self.boundary_conditions = MappingProxyType(dict(boundary_conditions))
        self.reference = build_reference_triangle(DEGREE)
        # the kernels' mesh tables are built by the GPU (cfd_mesh_build); the
        # host connectivity and geometry are computed when first asked for
        self._tables = DeviceTables.build_on_device(mesh, self.boundary_conditions, self.reference, device,
                                                    _native.CFD_FP64)
        self._finish_init(device, block_size, graph_chunk, variant)

    @property
    def connectivity(self):
        """Face connectivity (mesh.py:115-185 of CFD-demo), built on the host on first use."""
        conn = getattr(self, "_connectivity", None)
        if conn is None:
            conn = self._connectivity = build_connectivity(self.mesh)
        return conn

    @property
    def geometry(self):
        """Element geometry (mesh.py:188-243 of CFD-demo), computed on the host on first use."""
        geo = getattr(self, "_geometry", None)
        if geo is None:
            geo = self._geometry = element_geometry(self.mesh)
        return geo

    def _finish_init(self, device, block_size: int, graph_chunk: int, variant: int = 0) -> None:
        self.precision = PRECISIONS[self.config.precision]
        self.operators = self._tables.with_precision(self.precision)
        self._lib = _native.load()
        self._ws = Workspace(self.operators, self.precision, self.config.limiter != "unlimited")
        self._graph_chunk = int(graph_chunk)
        self._graphs: dict = {}
        self._struct = self._make_struct(block_size)
        self._struct.variant = int(variant)

    def with_precision(self, precision: str, **config_changes) -> "EulerSolver":
        """A solver on the same mesh and boundary conditions with another
        arithmetic form (and optionally other config fields), reusing the host
        setup."""
        import dataclasses

        other = object.__new__(EulerSolver)
        for name in ("mesh", "boundary_conditions", "reference", "_tables"):
            setattr(other, name, getattr(self, name))
        for name in ("_connectivity", "_geometry"):
            if hasattr(self, name):
                setattr(other, name, getattr(self, name))
        other.config = dataclasses.replace(self.config, precision=precision, **config_changes)
        other._finish_init(self.operators.device, self._struct.block_size, self._graph_chunk, self._struct.variant)
        return other

    # ---- native plumbing ------------------------------------------------------
    def _make_struct(self, block_size: int) -> _native.CfdSolver:
        ws = self._ws
        s = _native.CfdSolver()
        s.mesh = self.operators.struct
        s.flux = FLUX_IDS[self.config.flux]
        s.limiter = LIMITER_IDS[self.config.limiter]
        s.precision = self.precision
        s.max_rejections = self.config.max_rejections
        s.gamma = float(self.config.gamma)
        s.cfl = float(self.config.cfl)
        s.averages = ws.averages.data_ptr()
        s.element_aux = ws.aux.data_ptr()
        s.acc = ws.acc.data_ptr()
        s.report = ws.report.data_ptr()
        s.control = ws.control.data_ptr()
        s.limit_list = ws.limit_list.data_ptr()
        s.block_size = int(block_size)
        return s

    @property
    def native(self) -> _native.CfdSolver:
        """The CfdSolver struct handed to every C-ABI call."""
        return self._struct

    def set_block_size(self, block_size: int) -> None:
        self._struct.block_size = int(block_size)
        self._graphs.clear()

    def record_troubled_flags(self, enable: bool = True) -> None:
        """Have the limiter write its per-element troubled-cell indicator
        (limiting.py:147-151 of CFD-demo) on every call: stage k of a step
        writes row k-1 of :meth:`troubled_flags`, :meth:`limit` row 0."""
        self._struct.troubled_flags = self._ws.flags.data_ptr() if enable else None
        self._graphs.clear()

    def troubled_flags(self) -> np.ndarray:
        """(3, K) bool: the troubled-cell indicator of the last step's three
        stages (row 0 after :meth:`limit`); needs :meth:`record_troubled_flags`."""
        if not self._struct.troubled_flags:
            raise RuntimeError("troubled-flag recording is off; call record_troubled_flags() first.")
        return self._ws.flags[:, : self.mesh.num_elements].cpu().numpy().astype(bool)

    def set_variant(self, variant: int) -> None:
        """Select the stage-kernel variant (see CfdSolver.variant)."""
        self._struct.variant = int(variant)
        self._graphs.clear()

    @property
    def state_shape(self) -> tuple[int, int, int]:
        return (self.reference.num_nodes, self.mesh.num_elements, NUM_VARIABLES)

    @property
    def limiter_operators(self) -> LimiterOperators:
        """The limiter tables under the reference's names (solver.py:110 of
        CFD-demo builds them as a JAX pytree); host NumPy arrays here."""
        ops = getattr(self, "_limiter_operators", None)
        if ops is None:
            kind, state = resolve_boundary_conditions(self.connectivity, self.boundary_conditions)
            if (kind == EXACT_STATE).any():  # the ghost averages stand in for the exterior state
                ex = exact_state_rows(self.mesh, self.connectivity, self.reference, kind, self.boundary_conditions)
                state = state.copy()
                state[ex.elements, ex.faces] = ex.ghost
            ops = limiter_operators(self.connectivity, self.geometry, self.reference, kind, state)
            self._limiter_operators = ops
        return ops

    def node_coordinates(self) -> tuple[np.ndarray, np.ndarray]:
        """Physical node coordinates (x, y), each of shape (Np, K)."""
        return node_coordinates(self.mesh, self.reference.r, self.reference.s)

    def _as_state(self, q):
        import torch

        if isinstance(q, torch.Tensor):
            if tuple(q.shape) != self.state_shape:
                raise ValueError(f"Expected a state of shape {self.state_shape}, got {tuple(q.shape)}.")
            return q.to(device=self.operators.device, dtype=torch.float64, non_blocking=q.is_pinned()).contiguous()
        q = np.asarray(q, dtype=np.float64)
        if q.shape != self.state_shape:
            raise ValueError(f"Expected a state of shape {self.state_shape}, got {q.shape}.")
        return q

    def upload(self, q, out=None):
        """Host or device state (Np, K, 4) -> device layout tensor (60, ld)."""
        import torch

        q = self._as_state(q)
        if isinstance(q, np.ndarray):
            q = torch.from_numpy(np.ascontiguousarray(q)).to(self.operators.device, non_blocking=False)
        if out is None:
            out = torch.zeros((60, self.operators.ld), dtype=self._ws.dtype, device=self.operators.device)
        _native.check(self._lib.cfd_pack_state(q.data_ptr(), out.data_ptr(), self.mesh.num_elements,
                                               self.operators.ld, self.precision, _stream()))
        return out

    def download(self, x) -> np.ndarray:
        """Device layout tensor -> host (Np, K, 4) float64."""
        import torch

        tmp = torch.empty(self.state_shape, dtype=torch.float64, device=self.operators.device)
        _native.check(self._lib.cfd_unpack_state(x.data_ptr(), tmp.data_ptr(), self.mesh.num_elements,
                                                 self.operators.ld, self.precision, _stream()))
        # into page-locked memory (several times the bandwidth of a pageable
        # copy); the returned array owns its buffer (torch's host cache reuses
        # the pages once the array is gone)
        host = torch.empty(self.state_shape, dtype=torch.float64, pin_memory=True)
        host.copy_(tmp, non_blocking=True)
        torch.cuda.current_stream().synchronize()
        return host.numpy()

    def _write_control(self, **fields) -> None:
        import torch

        c = _native.CfdControl()
        for k, v in fields.items():
            setattr(c, k, v)
        buf = torch.frombuffer(bytearray(bytes(c)), dtype=torch.uint8)
        self._ws.control[: buf.numel()].copy_(buf)

    def _read(self, tensor, ctype, index: int = 0):
        raw = tensor.cpu().numpy().tobytes()
        size = C.sizeof(ctype)
        return ctype.from_buffer_copy(raw[index * size:(index + 1) * size])

    # ---- reference API (solver.py:141-165) -------------------------------------
    def rhs(self, q) -> tuple[np.ndarray, np.ndarray]:
        """Semi-discrete right-hand side and net outward boundary flux (dg.py:140-165)."""
        ws = self._ws
        x = self.upload(q, ws.x0)
        _native.check(self._lib.cfd_rhs(C.byref(self._struct), x.data_ptr(), ws.out.data_ptr(),
                                        ws.small.data_ptr(), _stream()))
        return self.download(ws.out), ws.small[:4].cpu().numpy().copy()

    def limit(self, q) -> np.ndarray:
        """Apply the troubled-cell and positivity limiters once (limiting.py:203-216)."""
        ws = self._ws
        x = self.upload(q, ws.x0)
        _native.check(self._lib.cfd_limit(C.byref(self._struct), x.data_ptr(), ws.out.data_ptr(),
                                          ws.small_i.data_ptr(), _stream()))
        return self.download(ws.out)

    def limit_with_count(self, q) -> tuple[np.ndarray, int]:
        ws = self._ws
        x = self.upload(q, ws.x0)
        _native.check(self._lib.cfd_limit(C.byref(self._struct), x.data_ptr(), ws.out.data_ptr(),
                                          ws.small_i.data_ptr(), _stream()))
        return self.download(ws.out), int(ws.small_i[0].item())

    def limit_with_flags(self, q) -> tuple[np.ndarray, np.ndarray]:
        """limit() plus the troubled-cell indicator of every element, (K,) bool."""
        ws = self._ws
        was = self._struct.troubled_flags
        self._struct.troubled_flags = ws.flags.data_ptr()
        try:
            x = self.upload(q, ws.x0)
            _native.check(self._lib.cfd_limit(C.byref(self._struct), x.data_ptr(), ws.out.data_ptr(),
                                              ws.small_i.data_ptr(), _stream()))
            flags = ws.flags[0, : self.mesh.num_elements].cpu().numpy().astype(bool)
        finally:
            self._struct.troubled_flags = was
        return self.download(ws.out), flags

    def time_step(self, q) -> float:
        """CFL time step for the state q (time_integration.py:37-41)."""
        ws = self._ws
        x = self.upload(q, ws.x0)
        _native.check(self._lib.cfd_time_step(C.byref(self._struct), x.data_ptr(), ws.small.data_ptr(), _stream()))
        return float(ws.small[0].item())

    def step(self, q, dt: float) -> tuple[np.ndarray, StepReport]:
        """One SSP-RK3 step without rejection handling (time_integration.py:44-84)."""
        ws = self._ws
        self.upload(q, ws.x0)
        self._write_control(dt=float(dt), final_time=np.inf, status=_native.RUN_ACTIVE, parity=0)
        _native.check(self._lib.cfd_rk3_attempt(C.byref(self._struct), ws.x0.data_ptr(), ws.x1.data_ptr(),
                                                ws.stage.data_ptr(), _stream()))
        rep = self._read(ws.report, _native.CfdStepReport)
        return self.download(ws.x1), self._report(rep)

    @staticmethod
    def _report(rep: _native.CfdStepReport) -> StepReport:
        return StepReport(boundary_flux=np.array(rep.boundary_flux[:]), admissible=bool(rep.admissible),
                          min_density=float(rep.min_density), min_pressure=float(rep.min_pressure),
                          troubled_cells=int(rep.troubled_cells))

    def cell_averages(self, q) -> np.ndarray:
        """Exact cell averages, shape (K, 4) (dg.py:168-171)."""
        ws = self._ws
        x = self.upload(q, ws.x0)
        _native.check(self._lib.cfd_cell_averages(C.byref(self._struct), x.data_ptr(), ws.averages.data_ptr(), _stream()))
        return ws.averages[:, : self.mesh.num_elements].T.cpu().numpy().copy()

    def integrate(self, q) -> np.ndarray:
        """Domain integral of each conserved variable, shape (4,) (dg.py:174-176)."""
        ws = self._ws
        x = self.upload(q, ws.x0)
        _native.check(self._lib.cfd_integrate(C.byref(self._struct), x.data_ptr(), ws.small.data_ptr(), _stream()))
        return ws.small[:4].cpu().numpy().copy()

    # ---- run loop (solver.py:167-216) ---------------------------------------------
    def _attempt_and_control(self, stream) -> None:
        ws = self._ws
        _native.check(self._lib.cfd_rk3_attempt(C.byref(self._struct), ws.x0.data_ptr(), ws.x1.data_ptr(),
                                                ws.stage.data_ptr(), stream))
        _native.check(self._lib.cfd_run_control(C.byref(self._struct), stream))

    def _chunk_graph(self, n: int):
        import torch

        g = self._graphs.get(n)
        if g is None:
            side = torch.cuda.Stream()
            side.wait_stream(torch.cuda.current_stream())
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g, stream=side):
                s = torch.cuda.current_stream().cuda_stream
                for _ in range(n):
                    self._attempt_and_control(s)
            torch.cuda.current_stream().wait_stream(side)
            self._graphs[n] = g
        return g

    def begin_run(self, initial_state, final_time: float) -> None:
        """Upload the state, check it (solver.py:170-176) and initialise the
        device-side loop state."""
        import torch

        ws = self._ws
        self.upload(initial_state, ws.x0)
        _native.check(self._lib.cfd_check_state(C.byref(self._struct), ws.x0.data_ptr(), ws.small.data_ptr(), _stream()))
        rmin, pmin, finite = (float(v) for v in ws.small[:3].cpu().numpy())
        if not (finite == 1.0 and rmin > 0.0 and pmin > 0.0):
            raise SolverError("The initial state must be finite with positive nodal density and pressure.")
        ft = torch.tensor([float(final_time)], dtype=torch.float64, device=self.operators.device)
        _native.check(self._lib.cfd_run_init(C.byref(self._struct), ws.x0.data_ptr(), ft.data_ptr(), _stream()))
        torch.cuda.current_stream().synchronize()

    def advance(self, attempts: int, *, graph: bool = True) -> _native.CfdControl:
        """Run `attempts` attempt+control passes (no-ops once the run ended) and
        return the device loop state."""
        if graph:
            self._chunk_graph(attempts).replay()
        else:
            s = _stream()
            for _ in range(attempts):
                self._attempt_and_control(s)
        return self._read(self._ws.control, _native.CfdControl)

    def state_tensor(self):
        """Current device state (device layout) of the run in progress."""
        c = self._read(self._ws.control, _native.CfdControl)
        return self._ws.x1 if c.parity else self._ws.x0

    def run(self, initial_state, final_time: float, *, graph: bool = True) -> RunResult:
        """Advance ``initial_state`` from t = 0 to ``final_time`` (solver.py:167-216)."""
        start = time.perf_counter()
        self.begin_run(initial_state, final_time)
        chunk = 1
        while True:
            c = self.advance(chunk, graph=graph)
            if c.status != _native.RUN_ACTIVE:
                break
            chunk = min(2 * chunk, self._graph_chunk)
        if c.status == _native.RUN_BAD_DT:
            raise SolverError(f"Invalid time step {c.dt} at t = {c.time}.")
        if c.status == _native.RUN_REJECTED:
            raise SolverError(f"Step at t = {c.time} was rejected {self.config.max_rejections + 1} times.")
        state = self.download(self._ws.x1 if c.parity else self._ws.x0)
        return RunResult(state=state, time=float(c.time), steps=int(c.steps), rejected_steps=int(c.rejected),
                         boundary_flux_integral=np.array(c.flux_integral[:]), min_density=float(c.min_density),
                         min_pressure=float(c.min_pressure), max_troubled_cells=int(c.max_troubled),
                         wall_time=time.perf_counter() - start)
