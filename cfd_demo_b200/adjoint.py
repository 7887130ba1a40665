"""Gradients of a fixed-schedule run: the hand-written discrete adjoint.

CFD-demo differentiates its step with ``jax.grad`` (its fluxes and limiters
are written to stay differentiable, fluxes.py:7 and limiters.py:4) and turns
each step size into a host float (solver.py:181), so the gradient of a run is
that of the composition of SSP-RK3 steps with the step sizes held fixed. The
same holds here: ``AdjointRun`` advances a state through a given schedule of
step sizes with ``cfd_rk3_step_fixed`` and back-propagates an adjoint through
the steps with ``cfd_rk3_step_adjoint`` (transposed Dr/Ds/LIFT, flux
Jacobian-transpose products, limiter branches replayed as taken).

Memory: the forward pass keeps one state every ``checkpoint_every`` steps; the
backward pass re-runs each segment from its checkpoint with the tape switched
on, then walks it in reverse. Peak device memory is about
``checkpoint_every * (6 states + 18 doubles per element)`` plus the
checkpoints.

``differentiable_run(runner, q0, bc_states)`` wraps this in a
``torch.autograd.Function``: q0 (Np, K, 4) and the fixed exterior states
(rows, 4) are differentiable inputs, the final state (Np, K, 4) the output.
"""

from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _native
from .solver import EulerSolver, SolverError, _stream


class AdjointRun:
    """Fixed-schedule run of ``solver`` and its discrete adjoint."""

    def __init__(self, solver: EulerSolver, dts, *, checkpoint_every: int = 20, hold_theta: bool = False):
        import torch

        if checkpoint_every < 1:
            raise ValueError("checkpoint_every must be at least 1.")
        self.solver = solver
        self.ops = solver.operators
        self._lib = solver._lib
        dts = np.asarray(dts, dtype=np.float64)
        if dts.ndim == 1:
            dts = dts[:, None]
        if dts.ndim != 2 or dts.shape[1] != self.ops.num_instances or dts.shape[0] < 1:
            raise ValueError(f"dts must have shape (steps,) or (steps, {self.ops.num_instances}).")
        if not np.all(np.isfinite(dts)) or np.any(dts <= 0.0):
            raise ValueError("Every step size must be finite and positive.")
        self.steps = dts.shape[0]
        self.dts = torch.from_numpy(dts.copy()).to(self.ops.device)
        self.checkpoint_every = int(checkpoint_every)
        # positivity limiter's bisection theta: implicit derivative (default) or
        # held constant, the derivative jax.grad takes of the bisection loop
        self.hold_theta = bool(hold_theta)
        ld, prec = self.ops.ld, solver.precision
        self._state_shape = (60, ld)
        self._tape_bytes = int(self._lib.cfd_tape_bytes(ld, prec))
        self._work = torch.empty(int(self._lib.cfd_adjoint_work_bytes(ld, prec)), dtype=torch.uint8,
                                 device=self.ops.device)
        self._stage = torch.zeros(self._state_shape, dtype=solver._ws.dtype, device=self.ops.device)

    # ---- plumbing ------------------------------------------------------------
    def _new_state(self):
        import torch

        return torch.zeros(self._state_shape, dtype=self.solver._ws.dtype, device=self.ops.device)

    def _dt(self, i: int) -> int:
        return self.dts.data_ptr() + 8 * i * self.ops.num_instances

    def _step(self, x_in, x_out, i: int, tape=None) -> None:
        _native.check(self._lib.cfd_rk3_step_fixed(C.byref(self.solver.native), x_in.data_ptr(), x_out.data_ptr(),
                                                   self._stage.data_ptr(), self._dt(i),
                                                   None if tape is None else tape.data_ptr(), _stream()))

    def pack(self, q):
        """(Np, K, 4) float64 device tensor -> device layout (the adjoint of unpack)."""
        import torch

        q = q.detach().to(device=self.ops.device, dtype=torch.float64).contiguous()
        out = self._new_state()
        _native.check(self._lib.cfd_pack_state(q.data_ptr(), out.data_ptr(), self.ops.num_elements, self.ops.ld,
                                               self.solver.precision, _stream()))
        return out

    def unpack(self, x):
        """Device layout -> (Np, K, 4) float64 device tensor (the adjoint of pack)."""
        import torch

        out = torch.empty(self.solver.state_shape, dtype=torch.float64, device=self.ops.device)
        _native.check(self._lib.cfd_unpack_state(x.data_ptr(), out.data_ptr(), self.ops.num_elements, self.ops.ld,
                                                 self.solver.precision, _stream()))
        return out

    def set_boundary_states(self, bc_states) -> None:
        """Overwrite the fixed exterior states (rows, 4) the kernels read."""
        import torch

        bc = torch.as_tensor(bc_states, dtype=torch.float64).to(self.ops.device).reshape(self.ops.bc_states.shape)
        self.ops.bc_states.copy_(bc)

    # ---- forward / backward ----------------------------------------------------
    def forward(self, x0):
        """Advance x0 (device layout) through the schedule. Returns the final
        state and the checkpoints {step: state}."""
        cur, nxt = x0.clone(), self._new_state()
        checkpoints = {0: x0.clone()}
        for i in range(self.steps):
            self._step(cur, nxt, i)
            cur, nxt = nxt, cur
            if (i + 1) % self.checkpoint_every == 0 and i + 1 < self.steps:
                checkpoints[i + 1] = cur.clone()
        return cur, checkpoints

    def backward(self, g_final, checkpoints, *, with_boundary: bool = True):
        """Adjoint of the final state (device layout) -> adjoint of the initial
        state (device layout) and of the fixed exterior states (rows, 4)."""
        import torch

        dev = self.ops.device
        bc_bar = torch.zeros(self.ops.bc_states.shape, dtype=torch.float64, device=dev)
        n = self.checkpoint_every
        seg_states = [self._new_state() for _ in range(n)]
        tapes = torch.empty((n, self._tape_bytes), dtype=torch.uint8, device=dev)
        out = self._new_state()
        g, g_next = g_final.clone(), self._new_state()
        starts = list(range(0, self.steps, n))
        for start in reversed(starts):
            stop = min(start + n, self.steps)
            seg_states[0].copy_(checkpoints[start])
            for i in range(start, stop):
                j = i - start
                dst = seg_states[j + 1] if j + 1 < n and i + 1 < stop else out
                self._step(seg_states[j], dst, i, tapes[j])
            for i in reversed(range(start, stop)):
                j = i - start
                _native.check(self._lib.cfd_rk3_step_adjoint(
                    C.byref(self.solver.native), seg_states[j].data_ptr(), tapes[j].data_ptr(), self._dt(i),
                    g.data_ptr(), g_next.data_ptr(), bc_bar.data_ptr() if with_boundary else None,
                    _native.ADJ_HOLD_THETA if self.hold_theta else 0, self._work.data_ptr(), _stream()))
                g, g_next = g_next, g
        return g, bc_bar


def cfl_schedule(solver: EulerSolver, q0, *, steps: int | None = None, final_time: float | None = None) -> np.ndarray:
    """Step sizes of the reference's run loop (solver.py:180-204) from q0: the
    CFL step of each state, clipped to the final time, halved on rejection.
    Stops after ``steps`` steps or at ``final_time``."""
    import torch

    if steps is None and final_time is None:
        raise ValueError("Give steps or final_time.")
    runner = AdjointRun(solver, [1.0], checkpoint_every=1)
    x = runner.pack(torch.as_tensor(np.asarray(q0, dtype=np.float64)))
    y = runner._new_state()
    dts, t = [], 0.0
    lib, s = solver._lib, solver.native
    ws = solver._ws
    dt_dev = torch.zeros(1, dtype=torch.float64, device=runner.ops.device)
    while (steps is None or len(dts) < steps) and (final_time is None or t < final_time):
        _native.check(lib.cfd_time_step(C.byref(s), x.data_ptr(), ws.small.data_ptr(), _stream()))
        dt = float(ws.small[0].item())
        if not math.isfinite(dt) or dt <= 0.0:
            raise SolverError(f"Invalid time step {dt} at t = {t}.")
        reaches_end = final_time is not None and dt >= final_time - t
        if reaches_end:
            dt = final_time - t
        for _ in range(solver.config.max_rejections + 1):
            dt_dev.fill_(dt)
            _native.check(lib.cfd_rk3_step_fixed(C.byref(s), x.data_ptr(), y.data_ptr(), runner._stage.data_ptr(),
                                                 dt_dev.data_ptr(), None, _stream()))
            if solver._read(ws.report, _native.CfdStepReport).admissible:
                break
            reaches_end = False
            dt *= 0.5
        else:
            raise SolverError(f"Step at t = {t} was rejected {solver.config.max_rejections + 1} times.")
        x, y = y, x
        t = final_time if reaches_end else t + dt
        dts.append(dt)
    return np.asarray(dts)


def _autograd_function():
    import torch

    class _Run(torch.autograd.Function):
        @staticmethod
        def forward(ctx, q0, bc_states, runner):
            runner.set_boundary_states(bc_states)
            x_final, checkpoints = runner.forward(runner.pack(q0))
            ctx.runner = runner
            ctx.checkpoints = checkpoints
            ctx.bc_states = bc_states.detach().clone()
            return runner.unpack(x_final)

        @staticmethod
        def backward(ctx, grad_out):
            runner = ctx.runner
            runner.set_boundary_states(ctx.bc_states)
            g0, bc_bar = runner.backward(runner.pack(grad_out), ctx.checkpoints,
                                         with_boundary=ctx.needs_input_grad[1])
            return runner.unpack(g0), bc_bar if ctx.needs_input_grad[1] else None, None

    return _Run


_RUN = None


def differentiable_run(runner: AdjointRun, q0, bc_states=None):
    """Final state (Np, K, 4) of ``runner``'s schedule from q0, differentiable
    in q0 and in the fixed exterior states ``bc_states`` (rows, 4; the
    solver's own when None) through torch.autograd."""
    import torch

    global _RUN
    if _RUN is None:
        _RUN = _autograd_function()
    if bc_states is None:
        bc_states = runner.ops.bc_states.clone()
    return _RUN.apply(q0, bc_states, runner)


def boundary_rows(solver: EulerSolver) -> dict:
    """Row of the fixed exterior-state table used by each FixedState tag."""
    rows = {}
    table = solver.operators.bc_states.cpu().numpy()
    for tag, bc in solver.boundary_conditions.items():
        state = getattr(bc, "state", None)
        if state is None:
            continue
        hit = np.flatnonzero(np.all(table == np.asarray(state, dtype=np.float64)[None], axis=1))
        if hit.size:
            rows[tag] = int(hit[0])
    return rows


class SodSensitivity:
    """Sensitivity study on the Sod tube: the left density rho_L is a
    parameter, a Gaussian density bump amplitude * exp(-((x - x_b) / width)^2)
    with x_b drawn from a seed in [0.2, 0.8] is added to the initial density,
    and the objective is J = sum over nodes of rho(T) * exp(-((x - 0.7) / width)^2).
    The left density enters both the initial state of the elements left of
    x = 0.5 and the fixed exterior state of the left boundary."""

    def __init__(self, nx: int = 400, ny: int = 40, *, flux: str = "rusanov", limiter: str = "minmod",
                 precision: str = "fp64", seed: int = 0, amplitude: float = 0.01, width: float = 0.05,
                 target: float = 0.7, bump_center: float | None = None, **solver_options):
        import torch

        from .cases import SOD_DISCONTINUITY, SOD_GAMMA, SOD_LEFT, SOD_RIGHT, sod_shock_tube

        case = sod_shock_tube(nx, ny, flux=flux, limiter=limiter, precision=precision, **solver_options)
        self.solver = case.solver
        self.gamma = SOD_GAMMA
        rng = np.random.default_rng(seed)
        drawn = float(rng.uniform(0.2, 0.8))
        self.bump_center = drawn if bump_center is None else float(bump_center)
        self.amplitude = amplitude
        x, _ = self.solver.node_coordinates()
        dev = self.solver.operators.device
        self.x = torch.from_numpy(x).to(dev)
        self.left = torch.from_numpy(self.solver.geometry.centroid[:, 0] < SOD_DISCONTINUITY).to(dev)
        self.bump = amplitude * torch.exp(-(((self.x - self.bump_center) / width) ** 2))
        self.weight = torch.exp(-(((self.x - target) / width) ** 2))
        self.right_state = torch.tensor(case.initial_state[0, ~self.left.cpu().numpy()][0], dtype=torch.float64,
                                        device=dev) if (~self.left).any() else None
        self.left_pressure = SOD_LEFT[3]
        self.rows = boundary_rows(self.solver)
        self.rho_left = SOD_LEFT[0]
        self._right_primitive = SOD_RIGHT

    def initial_state(self, rho_left):
        """(Np, K, 4) initial state as a differentiable function of rho_L."""
        import torch

        e_left = self.left_pressure / (self.gamma - 1.0)
        zero = torch.zeros_like(rho_left)
        left = torch.stack([rho_left, zero, zero, zero + e_left])
        q = torch.where(self.left[None, :, None], left[None, None, :], self.right_state[None, None, :])
        q = q.expand(self.x.shape[0], -1, -1)
        return q + torch.stack([self.bump, torch.zeros_like(self.bump), torch.zeros_like(self.bump),
                                torch.zeros_like(self.bump)], dim=-1)

    def boundary_states(self, rho_left):
        """Fixed exterior-state table with the left row depending on rho_L."""
        import torch

        base = self.solver.operators.bc_states.clone()
        row = self.rows["left"]
        e_left = self.left_pressure / (self.gamma - 1.0)
        zero = torch.zeros_like(rho_left)
        left = torch.stack([rho_left, zero, zero, zero + e_left])
        mask = torch.zeros(base.shape[0], 1, dtype=torch.float64, device=base.device)
        mask[row] = 1.0
        return base * (1.0 - mask) + mask * left[None, :]

    def objective(self, q):
        return (q[..., 0] * self.weight).sum()
