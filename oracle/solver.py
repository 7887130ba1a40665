"""Oracle: DG operator, limiters, SSP-RK3 step, CFL time step and run loop
(test infrastructure only).

Restates ``src/cfd_demo/dg.py``, ``limiting.py``, ``time_integration.py``,
``solver.py`` and ``cases.py`` of CFD-demo in NumPy float64, state layout
(Np, K, 4). ``OracleSolver`` offers the same methods as the reference's
``EulerSolver`` (rhs, limit, time_step, step, cell_averages, integrate, run).
"""

from __future__ import annotations

import time
from dataclasses import dataclass
from typing import NamedTuple

import numpy as np

from .element import DEGREE, build_reference_triangle
from .mesh import build_connectivity, element_geometry, node_coordinates, pair_face_nodes, rectangle_mesh
from .physics import (
    EXACT_STATE,
    FIXED_STATE,
    SLIP_WALL,
    FixedState,
    SlipWall,
    cartesian_fluxes,
    get_interface_flux,
    get_limiter_function,
    pressure,
    primitive_to_conserved,
    sound_speed,
    conserved_to_primitive,
)

# limiting.py:22-31
NEIGHBOR_FACTOR = 1.5
DETECTION_TOLERANCE = 1e-10
DETECTION_COMPONENTS = (0, 3)
POSITIVITY_FLOOR = 1e-13
BISECTION_STEPS = 60
_COEFF_TOL = 1e-12
# time_integration.py:18-19
DEFAULT_CFL = 0.5
MAX_REJECTIONS = 10


class SolverError(RuntimeError):
    """solver.py:33-34."""


class StepReport(NamedTuple):
    """time_integration.py:22-29."""

    boundary_flux: np.ndarray
    admissible: bool
    min_density: float
    min_pressure: float
    troubled_cells: int


@dataclass(frozen=True, eq=False)
class RunResult:
    """solver.py:62-88."""

    state: np.ndarray
    time: float
    steps: int
    rejected_steps: int
    boundary_flux_integral: np.ndarray
    min_density: float
    min_pressure: float
    max_troubled_cells: int
    wall_time: float


def mirror_state(q, nx, ny):
    """Slip-wall mirror: reverse the normal momentum (dg.py:119-126)."""
    mn = q[..., 1] * nx + q[..., 2] * ny
    z = np.zeros_like(mn)
    return q - np.stack([z, 2.0 * mn * nx, 2.0 * mn * ny, z], axis=-1)


def _minmod2(a, b):
    """limiting.py:124-125."""
    return np.where(a * b > 0.0, np.sign(a) * np.minimum(np.abs(a), np.abs(b)), 0.0)


class OracleSolver:
    """CPU restatement of ``EulerSolver`` (solver.py:91-216)."""

    def __init__(self, mesh, boundary_conditions, *, flux, limiter, gamma, cfl=DEFAULT_CFL,
                 max_rejections=MAX_REJECTIONS):
        get_interface_flux(flux)
        get_limiter_function(limiter)
        self.mesh = mesh
        self.flux_name, self.limiter_name = flux, limiter
        self.flux = get_interface_flux(flux)
        self.phi = get_limiter_function(limiter)
        self.limit_slopes = limiter != "unlimited"
        self.gamma, self.cfl, self.max_rejections = float(gamma), float(cfl), int(max_rejections)
        self.reference = ref = build_reference_triangle(DEGREE)
        self.connectivity = conn = build_connectivity(mesh)
        self.geometry = geo = element_geometry(mesh)
        k = mesh.num_elements
        nfp = ref.num_face_nodes

        # dg.py:52-73 — per-face boundary kinds and fixed states
        tags = set(conn.boundary_tags)
        if tags - set(boundary_conditions):
            raise ValueError(f"Boundary tags without a boundary condition: {sorted(tags - set(boundary_conditions))}.")
        if set(boundary_conditions) - tags:
            raise ValueError(f"Boundary conditions for tags that are not in the mesh: {sorted(set(boundary_conditions) - tags)}.")
        kind = np.zeros((k, 3), dtype=np.int32)
        state = np.zeros((k, 3, 4))
        for ti, tag in enumerate(conn.boundary_tags):
            bc = boundary_conditions[tag]
            m = conn.face_tag == ti
            kind[m] = bc.kind
            if bc.kind == FIXED_STATE:
                state[m] = bc.state
        self.boundary_kind, self.boundary_state = kind, state

        # dg.py:76-116 — operator arrays in face-node layout (3 Nfp, K)
        x, y = node_coordinates(mesh, ref.r, ref.s)
        # proposed ADR 0012: exact-state faces take per-node exterior states and
        # the reflected element's average as the ghost average
        node_state = np.zeros((3, nfp, k, 4))
        for ti, tag in enumerate(conn.boundary_tags):
            bc = boundary_conditions[tag]
            if bc.kind != EXACT_STATE:
                continue
            es, fs = np.nonzero(conn.face_tag == ti)
            for e, f in zip(es, fs):
                nodes = ref.face_nodes[f]
                node_state[f, :, e] = np.asarray(bc.function(x[nodes, e], y[nodes, e]), dtype=np.float64)
                state[e, f] = self._ghost_average(bc, mesh, e, f)
        partner = pair_face_nodes(mesh, conn, x, y, ref.face_nodes)
        own = np.arange(k)[:, None]
        nbr = np.where(conn.neighbor_element >= 0, conn.neighbor_element, own)

        def per_node(vals):  # (K, 3, ...) -> (3 Nfp, K, ...)
            vals = np.moveaxis(vals, 1, 0)[:, None]
            return np.broadcast_to(vals, (3, nfp) + vals.shape[2:]).reshape((3 * nfp,) + vals.shape[2:])

        self.face_nodes = ref.face_nodes.reshape(-1)
        self.nx = per_node(geo.normal[..., 0])
        self.ny = per_node(geo.normal[..., 1])
        self.fscale = per_node(0.5 * geo.edge_length / geo.jacobian[:, None])
        self.exterior_index = (partner * k + nbr.T[:, None, :]).reshape(3 * nfp, k)
        self.kind_fn = per_node(kind)
        self.state_fn = np.where((self.kind_fn == EXACT_STATE)[..., None], node_state.reshape(3 * nfp, k, 4),
                                 per_node(state))
        ew = ref.face_weights.reshape(-1)[:, None] * per_node(0.5 * geo.edge_length)
        self.bweight = np.where(self.kind_fn > 0, ew, 0.0)
        self.dmat = np.concatenate([ref.dr, ref.ds], axis=1)

        # limiting.py:51-121 — Cockburn-Shu coefficients and limiter tables
        self.alpha, self.beta, self.partner_face = self._cs_coefficients()
        self.avg_weights = ref.cell_weights / ref.cell_weights.sum()
        self.nbr3 = nbr.T  # (3, K)
        self.kind3 = kind.T
        self.nx3 = geo.normal[..., 0].T
        self.ny3 = geo.normal[..., 1].T
        self.fixed3 = np.moveaxis(state, 1, 0)
        # time_integration.py:32-34
        self.dt_geometry = np.min(2.0 * geo.area[:, None] / ((ref.degree + 1) ** 2 * geo.edge_length), axis=1)

    # ---- setup helpers -------------------------------------------------
    @staticmethod
    def _ghost_average(bc, mesh, e, f, subdivisions=32):
        """The exact-state function's average over element e reflected across
        its face f: bc.cell_average when given, else the mean over the
        centroids of subdivisions**2 equal sub-triangles."""
        c = mesh.vertices[mesh.elements[e]]
        a, b = c[f], c[(f + 1) % 3]
        d = b - a
        nrm = np.array([d[1], -d[0]]) / np.hypot(d[0], d[1])
        tri = c - 2.0 * ((c - a) @ nrm)[:, None] * nrm[None]
        if bc.cell_average is not None:
            return np.asarray(bc.cell_average(tri[None]), dtype=np.float64)[0]
        m = subdivisions
        pts = []
        for i in range(m):
            for j in range(m - i):
                pts.append(((i + 1 / 3) / m, (j + 1 / 3) / m))
                if i + j < m - 1:
                    pts.append(((i + 2 / 3) / m, (j + 2 / 3) / m))
        lam = np.array(pts)
        p = tri[0] + lam[:, :1] * (tri[1] - tri[0]) + lam[:, 1:] * (tri[2] - tri[0])
        return np.asarray(bc.function(p[:, 0], p[:, 1]), dtype=np.float64).mean(axis=0)

    def _cs_coefficients(self):
        """limiting.py:51-94."""
        geo, conn = self.geometry, self.connectivity
        cen, mid, nrm, nb = geo.centroid, geo.face_midpoint, geo.normal, conn.neighbor_element
        off = np.sum((mid - cen[:, None]) * nrm, axis=-1, keepdims=True)
        refl = cen[:, None] + 2.0 * off * nrm
        ncen = np.where((nb >= 0)[..., None], cen[np.maximum(nb, 0)], refl)
        d = ncen - cen[:, None]
        t = mid - cen[:, None]
        k = cen.shape[0]
        alpha, beta = np.zeros((k, 3)), np.zeros((k, 3))
        partner = -np.ones((k, 3), dtype=np.int64)
        for f in range(3):
            for shift in (1, 2):
                o = (f + shift) % 3
                di, dj, tt = d[:, f], d[:, o], t[:, f]
                det = di[:, 0] * dj[:, 1] - di[:, 1] * dj[:, 0]
                safe = np.where(det == 0.0, 1.0, det)
                a = (tt[:, 0] * dj[:, 1] - tt[:, 1] * dj[:, 0]) / safe
                b = (di[:, 0] * tt[:, 1] - di[:, 1] * tt[:, 0]) / safe
                ok = (det != 0.0) & (a >= -_COEFF_TOL) & (b >= -_COEFF_TOL) & (partner[:, f] < 0)
                alpha[ok, f] = np.maximum(a[ok], 0.0)
                beta[ok, f] = np.maximum(b[ok], 0.0)
                partner[ok, f] = o
        if np.any(partner < 0):
            e, f = np.argwhere(partner < 0)[0]
            raise ValueError(f"No nonnegative Cockburn-Shu neighbor coefficients for face {f} of element {e}.")
        return alpha.T, beta.T, partner.T

    # ---- public API (solver.py:127-165) ---------------------------------
    @property
    def state_shape(self):
        return (self.reference.num_nodes, self.mesh.num_elements, 4)

    def node_coordinates(self):
        return node_coordinates(self.mesh, self.reference.r, self.reference.s)

    def _as_state(self, q):
        q = np.asarray(q, dtype=np.float64)
        if q.shape != self.state_shape:
            raise ValueError(f"Expected a state of shape {self.state_shape}, got {q.shape}.")
        return q

    def rhs(self, q):
        """dg.py:140-165."""
        q = self._as_state(q)
        f, g = cartesian_fluxes(q, self.gamma)
        rx, ry, sx, sy = (a[None, :, None] for a in (self.geometry.rx, self.geometry.ry, self.geometry.sx, self.geometry.sy))
        contra = np.concatenate([rx * f + ry * g, sx * f + sy * g], axis=0)
        div = np.einsum("ij,jkc->ikc", self.dmat, contra)
        qm = q[self.face_nodes]
        qn = q.reshape(-1, 4)[self.exterior_index]
        kind = self.kind_fn[..., None]
        qp = np.where(kind == SLIP_WALL, mirror_state(qm, self.nx, self.ny),
                      np.where(kind >= FIXED_STATE, self.state_fn, qn))
        fhat = self.flux(qm, qp, self.nx, self.ny, self.gamma)
        fminus = f[self.face_nodes] * self.nx[..., None] + g[self.face_nodes] * self.ny[..., None]
        jump = self.fscale[..., None] * (fminus - fhat)
        surface = np.einsum("ij,jkc->ikc", self.reference.lift, jump)
        bflux = np.einsum("jk,jkc->c", self.bweight, fhat)
        return surface - div, bflux

    def _neighbor_averages(self, avg):
        """limiting.py:128-133."""
        interior = avg[self.nbr3]
        wall = mirror_state(avg[None], self.nx3, self.ny3)
        kind = self.kind3[..., None]
        return np.where(kind == SLIP_WALL, wall, np.where(kind >= FIXED_STATE, self.fixed3, interior))

    def troubled_cell_limit(self, q, avg):
        """limiting.py:136-163. Returns (limited q, troubled flags (K,))."""
        ref = self.reference
        diff = self._neighbor_averages(avg) - avg[None]
        paired = np.take_along_axis(diff, self.partner_face[..., None], axis=0)
        scaled = NEIGHBOR_FACTOR * (self.alpha[..., None] * diff + self.beta[..., None] * paired)
        trace = q[ref.face_midpoint_nodes] - avg[None]
        comp = list(DETECTION_COMPONENTS)
        excess = np.abs(_minmod2(trace, scaled) - trace)[..., comp]
        thresh = DETECTION_TOLERANCE * np.abs(avg[:, comp])
        troubled = np.any(excess > thresh[None], axis=(0, 2))
        proj = np.einsum("fi,ikc->fkc", ref.p1_midpoint, q) - avg[None]
        nz = proj != 0.0
        with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
            ratio = scaled / np.where(nz, proj, 1.0)
            deltas = np.where(nz, proj * np.minimum(1.0, self.phi(ratio)), 0.0)
            pos = np.sum(np.maximum(deltas, 0.0), axis=0)
            neg = np.sum(np.maximum(-deltas, 0.0), axis=0)
            th_p = np.where(pos > 0.0, np.minimum(1.0, neg / np.where(pos > 0.0, pos, 1.0)), 0.0)
            th_n = np.where(neg > 0.0, np.minimum(1.0, pos / np.where(neg > 0.0, neg, 1.0)), 0.0)
        deltas = th_p[None] * np.maximum(deltas, 0.0) - th_n[None] * np.maximum(-deltas, 0.0)
        linear = avg[None] + np.einsum("if,fkc->ikc", ref.linear_midpoint_basis, deltas)
        return np.where(troubled[None, :, None], linear, q), troubled

    def detection_ratios(self, q, avg):
        """The troubled-cell test of limiting.py:141-151 as one number per
        element: the largest excess / threshold over the three face midpoints
        and the detection components (troubled exactly when it exceeds one;
        inf where a threshold is zero and the excess is not). A ratio within
        round-off of one marks a decision that round-off can flip."""
        ref = self.reference
        diff = self._neighbor_averages(avg) - avg[None]
        paired = np.take_along_axis(diff, self.partner_face[..., None], axis=0)
        scaled = NEIGHBOR_FACTOR * (self.alpha[..., None] * diff + self.beta[..., None] * paired)
        trace = q[ref.face_midpoint_nodes] - avg[None]
        comp = list(DETECTION_COMPONENTS)
        excess = np.abs(_minmod2(trace, scaled) - trace)[..., comp]
        thresh = DETECTION_TOLERANCE * np.abs(avg[:, comp])[None]
        with np.errstate(divide="ignore", invalid="ignore"):
            ratio = np.where(thresh > 0, excess / thresh, np.where(excess > 0, np.inf, 0.0))
        return ratio.max(axis=(0, 2))

    def positivity_limit(self, q, avg):
        """limiting.py:166-200."""
        g = self.gamma
        rho_a = avg[:, 0]
        p_a = pressure(avg, g)
        eps = np.minimum(POSITIVITY_FLOOR, np.minimum(rho_a, p_a))
        dev = q - avg[None]
        rho_min = np.min(q[..., 0], axis=0)
        need_rho = rho_min < eps
        span = np.where(need_rho, rho_a - rho_min, 1.0)
        theta = np.clip(np.where(need_rho, (rho_a - eps) / span, 1.0), 0.0, 1.0)
        q = np.where(need_rho[None, :, None], avg[None] + theta[None, :, None] * dev, q)
        with np.errstate(invalid="ignore", divide="ignore"):
            need_p = pressure(q, g) < eps[None]
        if not np.any(need_p):
            return q
        dev = q - avg[None]
        lo, hi = np.zeros(q.shape[:2]), np.ones(q.shape[:2])
        for _ in range(BISECTION_STEPS):
            mid = 0.5 * (lo + hi)
            with np.errstate(invalid="ignore", divide="ignore"):
                ok = pressure(avg[None] + mid[..., None] * dev, g) >= eps[None]
            lo, hi = np.where(ok, mid, lo), np.where(ok, hi, mid)
        theta = np.min(np.where(need_p, lo, 1.0), axis=0)
        limited = avg[None] + theta[None, :, None] * dev
        return np.where((theta < 1.0)[None, :, None], limited, q)

    def apply_limiters(self, q):
        """limiting.py:203-216. Returns (q, averages, troubled_count, troubled flags)."""
        avg = np.einsum("i,ikc->kc", self.avg_weights, q)
        if self.limit_slopes:
            q, troubled = self.troubled_cell_limit(q, avg)
        else:
            troubled = np.zeros(q.shape[1], dtype=bool)
        q = self.positivity_limit(q, avg)
        return q, avg, int(troubled.sum()), troubled

    def limit(self, q):
        return self.apply_limiters(self._as_state(q))[0]

    def time_step(self, q):
        """time_integration.py:37-41."""
        rho, u, v, p = conserved_to_primitive(self._as_state(q), self.gamma)
        with np.errstate(invalid="ignore"):
            lam = np.sqrt(u * u + v * v) + sound_speed(rho, p, self.gamma)
        return float(self.cfl * np.min(self.dt_geometry / np.max(lam, axis=0)))

    def step(self, q, dt, *, record=None, ratios=None):
        """time_integration.py:44-84. ``record``, if a list, receives the
        troubled flags of each stage; ``ratios``, if a list, each stage's
        detection_ratios of its state before limiting."""
        q = self._as_state(q)
        g = self.gamma

        def lim(u):
            if ratios is not None:
                ratios.append(self.detection_ratios(u, np.einsum("i,ikc->kc", self.avg_weights, u)))
            u, avg, count, flags = self.apply_limiters(u)
            if record is not None:
                record.append(flags)
            with np.errstate(invalid="ignore"):
                ok = bool(np.all(np.isfinite(u)) & np.all(avg[:, 0] > 0.0) & np.all(pressure(avg, g) > 0.0))
            return u, ok, count

        r0, b0 = self.rhs(q)
        q1, ok1, t1 = lim(q + dt * r0)
        r1, b1 = self.rhs(q1)
        q2, ok2, t2 = lim(0.75 * q + 0.25 * (q1 + dt * r1))
        r2, b2 = self.rhs(q2)
        q3, ok3, t3 = lim(q / 3.0 + 2.0 / 3.0 * (q2 + dt * r2))
        with np.errstate(invalid="ignore"):
            report = StepReport(
                boundary_flux=dt * (b0 / 6.0 + b1 / 6.0 + 2.0 * b2 / 3.0),
                admissible=ok1 and ok2 and ok3,
                min_density=float(min(np.min(s[..., 0]) for s in (q1, q2, q3))),
                min_pressure=float(min(np.min(pressure(s, g)) for s in (q1, q2, q3))),
                troubled_cells=max(t1, t2, t3),
            )
        return q3, report

    def cell_averages(self, q):
        """dg.py:168-171."""
        w = self.reference.cell_weights / np.sum(self.reference.cell_weights)
        return np.einsum("i,ikc->kc", w, self._as_state(q))

    def integrate(self, q):
        """dg.py:174-176."""
        return np.einsum("k,i,ikc->c", self.geometry.jacobian, self.reference.cell_weights, self._as_state(q))

    def run(self, initial_state, final_time, *, trace=None):
        """Host loop of solver.py:167-216. ``trace``, if a list, receives
        (dt, report) for every accepted step."""
        start = time.perf_counter()
        q = self._as_state(initial_state)
        p0 = pressure(q, self.gamma)
        if not (np.all(np.isfinite(q)) and np.all(q[..., 0] > 0.0) and np.all(p0 > 0.0)):
            raise SolverError("The initial state must be finite with positive nodal density and pressure.")
        min_rho, min_p = float(np.min(q[..., 0])), float(np.min(p0))
        flux_int = np.zeros(4)
        t, steps, rejected, max_tr = 0.0, 0, 0, 0
        while t < final_time:
            dt = self.time_step(q)
            if not np.isfinite(dt) or dt <= 0.0:
                raise SolverError(f"Invalid time step {dt} at t = {t}.")
            remaining = final_time - t
            reaches_end = dt >= remaining
            dt = remaining if reaches_end else dt
            for _ in range(self.max_rejections + 1):
                q_new, rep = self.step(q, dt)
                if rep.admissible:
                    break
                rejected += 1
                reaches_end = False
                dt *= 0.5
            else:
                raise SolverError(f"Step at t = {t} was rejected {self.max_rejections + 1} times.")
            q = q_new
            t = final_time if reaches_end else t + dt
            steps += 1
            flux_int += rep.boundary_flux
            min_rho = min(min_rho, rep.min_density)
            min_p = min(min_p, rep.min_pressure)
            max_tr = max(max_tr, rep.troubled_cells)
            if trace is not None:
                trace.append((dt, rep))
        return RunResult(q, t, steps, rejected, flux_int, min_rho, min_p, max_tr, time.perf_counter() - start)


# cases.py:15-44
SOD_GAMMA = 1.4
SOD_LEFT = (1.0, 0.0, 0.0, 1.0)
SOD_RIGHT = (0.125, 0.0, 0.0, 0.1)
SOD_FINAL_TIME = 0.2


def sod_shock_tube(nx=200, ny=20, *, flux, limiter, cfl=DEFAULT_CFL):
    """cases.py:31-44. Returns (solver, initial_state, final_time)."""
    mesh = rectangle_mesh(nx, ny, (0.0, 1.0), (0.0, 0.1))
    left = FixedState.from_primitive(*SOD_LEFT, gamma=SOD_GAMMA)
    right = FixedState.from_primitive(*SOD_RIGHT, gamma=SOD_GAMMA)
    bcs = {"left": left, "right": right, "bottom": SlipWall(), "top": SlipWall()}
    solver = OracleSolver(mesh, bcs, flux=flux, limiter=limiter, gamma=SOD_GAMMA, cfl=cfl)
    on_left = solver.geometry.centroid[:, 0] < 0.5
    es = np.where(on_left[:, None], np.array(left.state), np.array(right.state))
    return solver, np.broadcast_to(es[None], solver.state_shape).copy(), SOD_FINAL_TIME


__all__ = ["OracleSolver", "RunResult", "SolverError", "StepReport", "sod_shock_tube", "primitive_to_conserved"]
