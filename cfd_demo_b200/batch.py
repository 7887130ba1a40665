"""Many independent DG Euler problems advanced together on one GPU.

`BatchedEulerSolver` concatenates the meshes of several problems ("instances")
into one element range (each instance starting at a multiple of 64 elements)
so that every stage kernel launch covers all of them. Each instance keeps its
own run-loop state on the device (CfdControl: time, dt, parity of its state
buffers, step and rejection counts, minima, boundary-flux integral), so the
instances march with their own CFL steps, are rejected and retried on their
own, and stop at their own final time exactly as `EulerSolver.run` does
(solver.py:167-216 of CFD-demo); finished instances are skipped by the kernels.
Two execution forms. ``persistent=True`` (the default): each chunk of
attempts is ONE cooperative launch (cfd_batch_advance) whose blocks stay
resident, loop over the tiles of every instance and step through the phases
of each attempt with grid-wide barriers; the chunk's launch is captured in a
CUDA graph and replayed. ``persistent=False``: CUDA-graph chunks of the
separate launches (cfd_rk3_attempt + cfd_run_control per attempt). Either
way the host polls the loop states once per chunk. With ``compact=True``,
once the instances still running hold at most half of the batch's elements,
`run` / `run_to` repack them into a smaller batch (same tables, states and
loop states), so that the launches stop sweeping the tiles of finished
instances. Off by default: the blocks of finished instances exit at once, so
on the seeded family repacking bought nothing against its table uploads and
graph captures.

`riemann_batch` builds the seeded benchmark family: Riemann problems on
[0,1]x[0,0.1] strips split at x = 0.5 with left/right density and pressure
uniform in [0.1, 1], zero velocity, nx uniform in {50..400}, ny = floor(nx/10).
"""

from __future__ import annotations

import ctypes as C
import time
from dataclasses import dataclass

import numpy as np

from . import _native
from .boundary import FixedState, SlipWall
from .euler import NUM_VARIABLES
from .fluxes import FLUX_IDS
from .limiters import LIMITER_IDS
from .mesh import build_connectivity, element_geometry, rectangle_mesh
from .operators import DeviceTables, host_tables, resolve_boundary_conditions
from .reference_element import DEGREE, build_reference_triangle
from .solver import PRECISIONS, RunResult, SolverConfig, SolverError, Workspace, _stream


@dataclass(frozen=True, eq=False)
class BatchCase:
    mesh: object
    boundary_conditions: dict
    initial_state: np.ndarray


def riemann_batch(count: int = 256, seed: int = 0, nx_range=(50, 400), gamma: float = 1.4) -> list[BatchCase]:
    """Seeded Riemann problems on [0,1]x[0,0.1] (left/right rho, p in [0.1, 1],
    u = v = 0, split at x = 0.5), meshes nx x floor(nx/10) quads of 2 triangles."""
    rng = np.random.default_rng(seed)
    cases = []
    for _ in range(count):
        nx = int(rng.integers(nx_range[0], nx_range[1] + 1))
        ny = max(1, nx // 10)
        rl, rr, pl, pr = rng.uniform(0.1, 1.0, size=4)
        mesh = rectangle_mesh(nx, ny, (0.0, 1.0), (0.0, 0.1))
        left = FixedState.from_primitive(rl, 0.0, 0.0, pl, gamma)
        right = FixedState.from_primitive(rr, 0.0, 0.0, pr, gamma)
        bcs = {"left": left, "right": right, "bottom": SlipWall(), "top": SlipWall()}
        cen = mesh.vertices[mesh.elements].mean(axis=1)
        es = np.where((cen[:, 0] < 0.5)[:, None], np.array(left.state), np.array(right.state))
        q0 = np.broadcast_to(es[None], (15, mesh.num_elements, 4)).copy()
        cases.append(BatchCase(mesh, bcs, q0))
    return cases


class BatchedEulerSolver:
    """Several independent problems with one configuration, advanced together."""

    def __init__(self, cases, config: SolverConfig, *, device="cuda", graph_chunk: int = 64, variant: int = 0,
                 persistent: bool = True, compact: bool = False, _parts=None):
        import torch

        if not torch.cuda.is_available():
            raise RuntimeError("cfd_demo_b200 needs a CUDA GPU (B200); there is no CPU fallback.")
        self.config = config
        self.reference = build_reference_triangle(DEGREE)
        self.cases = list(cases)
        if _parts is None:
            parts = []
            for case in self.cases:
                conn = build_connectivity(case.mesh)
                geo = element_geometry(case.mesh)
                kind, state = resolve_boundary_conditions(conn, case.boundary_conditions)
                parts.append(host_tables(case.mesh, conn, geo, self.reference, kind, state, device=device,
                                         boundary_conditions=case.boundary_conditions))
        else:
            parts = list(_parts)
        self._parts = parts
        self._device = device
        self.compact = bool(compact)
        self.precision = PRECISIONS[config.precision]
        self.operators = DeviceTables(parts, device, self.precision)
        self._ws = Workspace(self.operators, self.precision, config.limiter != "unlimited")
        self._lib = _native.load()
        s = _native.CfdSolver()
        s.mesh = self.operators.struct
        s.flux = FLUX_IDS[config.flux]
        s.limiter = LIMITER_IDS[config.limiter]
        s.precision = self.precision
        s.max_rejections = config.max_rejections
        s.gamma = float(config.gamma)
        s.cfl = float(config.cfl)
        s.averages = self._ws.averages.data_ptr()
        s.element_aux = self._ws.aux.data_ptr()
        s.acc = self._ws.acc.data_ptr()
        s.report = self._ws.report.data_ptr()
        s.control = self._ws.control.data_ptr()
        s.variant = int(variant)
        s.limit_list = self._ws.limit_list.data_ptr()
        self._struct = s
        self._graph_chunk = int(graph_chunk)
        self._graphs: dict = {}
        self.persistent = bool(persistent)
        if self.persistent:  # the per-device lookup of the resident grid, outside any capture
            _native.check(self._lib.cfd_batch_advance(C.byref(s), self._ws.x0.data_ptr(), self._ws.x1.data_ptr(),
                                                      self._ws.stage.data_ptr(), 0, _stream()))

    @property
    def num_instances(self) -> int:
        return len(self.cases)

    @property
    def num_elements(self) -> int:
        return int(self.operators.sizes.sum())

    @property
    def native(self) -> _native.CfdSolver:
        return self._struct

    def set_variant(self, variant: int) -> None:
        self._struct.variant = int(variant)
        self._graphs.clear()

    def run_to(self, states, final_time, *, max_chunk: int | None = None, max_attempts: int | None = None) -> list:
        """Advance every instance from t = 0 until each has ended (done, or
        stopped by a bad CFL step or too many rejections, without raising),
        or `max_attempts` attempts have run (instances still active are left
        so); returns the loop states (CfdControl) of all instances."""
        where = self._march(states, final_time, max_chunk or self._graph_chunk, max_attempts, True)
        return [c for _, _, c in where]

    def _march(self, states, final_time, cap_chunk: int, max_attempts, graph: bool) -> list:
        """Begin a run and advance in chunks of attempts (1, 2, 4, ... up to
        cap_chunk) until no instance is active or max_attempts attempts have
        run. With `compact`, whenever the active instances hold at most half
        of the current batch's elements they are repacked into a smaller
        batch (`_subset`), so that the launches stop sweeping the tiles of
        finished instances. Returns per instance (batch holding its final
        state, its index there, its loop state)."""
        self.begin_run(states, final_time)
        cur, ids = self, list(range(self.num_instances))
        where: list = [None] * self.num_instances
        chunk, done = 1, 0
        while True:
            ctl = cur.advance(chunk, graph=graph)
            done += chunk
            for k, i in enumerate(ids):
                where[i] = (cur, k, ctl[k])
            active = [k for k, c in enumerate(ctl) if c.status == _native.RUN_ACTIVE]
            if not active or (max_attempts and done >= max_attempts):
                return where
            if cur.compact and len(active) < len(ctl):
                live = sum(int(cur.operators.sizes[k]) for k in active)
                if 2 * live <= cur.num_elements:
                    cur, ids = cur._subset(active, ctl), [ids[k] for k in active]
            chunk = min(2 * chunk, cap_chunk)

    def _subset(self, keep: list, ctl: list) -> "BatchedEulerSolver":
        """A batch of the instances `keep` (indices into this batch) that
        carries on from their current states and loop states (read at a chunk
        boundary). The tables are this batch's host tables (not rebuilt); each
        state is copied into the new batch's first buffer and its loop state's
        parity set to match. Tiles never straddle instances, so every element
        is computed exactly as it would have been in this batch."""
        import torch

        sub = BatchedEulerSolver([self.cases[i] for i in keep], self.config, device=self._device,
                                 graph_chunk=self._graph_chunk, variant=self._struct.variant,
                                 persistent=self.persistent, compact=self.compact,
                                 _parts=[self._parts[i] for i in keep])
        sub._struct.block_size = self._struct.block_size
        raw = bytearray()
        for k, i in enumerate(keep):
            c = _native.CfdControl.from_buffer_copy(bytes(ctl[i]))
            src = self._ws.x1 if c.parity else self._ws.x0
            o, n, on = int(self.operators.offsets[i]), int(self.operators.sizes[i]), int(sub.operators.offsets[k])
            sub._ws.x0[:, on:on + n].copy_(src[:, o:o + n])
            c.parity = 0
            raw += bytes(c)
        sub._ws.control.copy_(torch.frombuffer(raw, dtype=torch.uint8).to(sub._ws.control.device))
        return sub

    def set_block_size(self, block: int) -> None:
        self._struct.block_size = int(block)
        self._graphs.clear()

    def _elem_bytes(self) -> int:
        return 8 if self.precision == _native.CFD_FP64 else 4

    def upload(self, states, out=None):
        """Pack every instance's (Np, K_i, 4) state into one device buffer."""
        import torch

        ws = self._ws
        out = ws.x0 if out is None else out
        for i, q in enumerate(states):
            q = np.asarray(q, dtype=np.float64)
            k = int(self.operators.sizes[i])
            if q.shape != (15, k, NUM_VARIABLES):
                raise ValueError(f"Instance {i}: expected a state of shape {(15, k, 4)}, got {q.shape}.")
            t = torch.from_numpy(np.ascontiguousarray(q)).to(self.operators.device)
            ptr = out.data_ptr() + int(self.operators.offsets[i]) * self._elem_bytes()
            _native.check(self._lib.cfd_pack_state(t.data_ptr(), ptr, k, self.operators.ld, self.precision, _stream()))
        return out

    def download(self, x, i: int) -> np.ndarray:
        import torch

        k = int(self.operators.sizes[i])
        tmp = torch.empty((15, k, 4), dtype=torch.float64, device=self.operators.device)
        ptr = x.data_ptr() + int(self.operators.offsets[i]) * self._elem_bytes()
        _native.check(self._lib.cfd_unpack_state(ptr, tmp.data_ptr(), k, self.operators.ld, self.precision, _stream()))
        return tmp.cpu().numpy()

    def controls(self) -> list:
        raw = self._ws.control.cpu().numpy().tobytes()
        size = C.sizeof(_native.CfdControl)
        return [_native.CfdControl.from_buffer_copy(raw[i * size:(i + 1) * size]) for i in range(self.num_instances)]

    def begin_run(self, states, final_time) -> None:
        import torch

        ws = self._ws
        self.upload(states, ws.x0)
        n = self.num_instances
        _native.check(self._lib.cfd_check_state(C.byref(self._struct), ws.x0.data_ptr(), ws.small.data_ptr(), _stream()))
        chk = ws.small[: 3 * n].cpu().numpy().reshape(n, 3)
        bad = [i for i in range(n) if not (chk[i, 2] == 1.0 and chk[i, 0] > 0.0 and chk[i, 1] > 0.0)]
        if bad:
            raise SolverError(f"Instances {bad[:8]}: the initial state must be finite with positive nodal density and pressure.")
        ft = np.broadcast_to(np.asarray(final_time, dtype=np.float64), (n,)).copy()
        ftd = torch.from_numpy(ft).to(self.operators.device)
        _native.check(self._lib.cfd_run_init(C.byref(self._struct), ws.x0.data_ptr(), ftd.data_ptr(), _stream()))
        torch.cuda.current_stream().synchronize()

    def _attempt_and_control(self, stream) -> None:
        ws = self._ws
        _native.check(self._lib.cfd_rk3_attempt(C.byref(self._struct), ws.x0.data_ptr(), ws.x1.data_ptr(),
                                                ws.stage.data_ptr(), stream))
        _native.check(self._lib.cfd_run_control(C.byref(self._struct), stream))

    def _persistent_chunk(self, attempts: int, stream) -> None:
        ws = self._ws
        _native.check(self._lib.cfd_batch_advance(C.byref(self._struct), ws.x0.data_ptr(), ws.x1.data_ptr(),
                                                  ws.stage.data_ptr(), int(attempts), stream))

    def _issue(self, n: int, stream) -> None:
        if self.persistent:
            self._persistent_chunk(n, stream)
        else:
            for _ in range(n):
                self._attempt_and_control(stream)

    def _chunk_graph(self, n: int):
        import torch

        key = (n, self.persistent)
        g = self._graphs.get(key)
        if g is None:
            if self.persistent:  # the per-device lookup of the resident grid, outside the capture
                self._persistent_chunk(0, torch.cuda.current_stream().cuda_stream)
            side = torch.cuda.Stream()
            side.wait_stream(torch.cuda.current_stream())
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g, stream=side):
                self._issue(n, torch.cuda.current_stream().cuda_stream)
            torch.cuda.current_stream().wait_stream(side)
            self._graphs[key] = g
        return g

    def advance(self, attempts: int, *, graph: bool = True) -> list:
        """Run `attempts` attempt + control passes (no-ops for finished
        instances) and return every instance's loop state."""
        if graph:
            self._chunk_graph(attempts).replay()
        else:
            self._issue(attempts, _stream())
        return self.controls()

    def run(self, states=None, final_time=None, *, graph: bool = True) -> list[RunResult]:
        """Advance every instance from t = 0 to its final time; one RunResult
        per instance (same fields as EulerSolver.run)."""
        start = time.perf_counter()
        states = [c.initial_state for c in self.cases] if states is None else states
        where = self._march(states, final_time, self._graph_chunk, None, graph)
        ctl = [c for _, _, c in where]
        failed = [(i, c) for i, c in enumerate(ctl) if c.status not in (_native.RUN_DONE,)]
        if failed:
            i, c = failed[0]
            what = "invalid time step" if c.status == _native.RUN_BAD_DT else "too many rejections"
            raise SolverError(f"Instance {i} stopped at t = {c.time}: {what} ({len(failed)} instance(s) failed).")
        wall = time.perf_counter() - start
        out = []
        for b, k, c in where:
            x = b._ws.x1 if c.parity else b._ws.x0
            out.append(RunResult(state=b.download(x, k), time=float(c.time), steps=int(c.steps),
                                 rejected_steps=int(c.rejected), boundary_flux_integral=np.array(c.flux_integral[:]),
                                 min_density=float(c.min_density), min_pressure=float(c.min_pressure),
                                 max_troubled_cells=int(c.max_troubled), wall_time=wall))
        return out
