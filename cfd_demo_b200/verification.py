"""Verification diagnostics of Riemann-problem runs (the Sod tube), evaluated
with PyTorch on the GPU.

* ``ExactRiemann``: the exact solution of the 1D Riemann problem for an ideal
  gas (the star pressure by Newton iteration on the pressure function, then
  the self-similar wave fan: rarefaction or shock on each side, a contact in
  between), as in Toro, "Riemann Solvers and Numerical Methods for Fluid
  Dynamics", ch. 4.
* ``Quadrature``: integration points over a triangle mesh, with every element
  that a given vertical line x = x_b crosses cut along it, so that the exact
  solution's discontinuities fall on sub-triangle boundaries. Each piece uses
  a collapsed (Duffy) tensor Gauss-Legendre rule.
* ``evaluate``: the nodal degree-4 solution at the integration points
  (Lagrange basis from the orthonormal Vandermonde matrix), on the GPU.
* ``l1_errors``, ``column_density`` / ``front_position``: the domain-averaged
  L1 errors against the exact solution and the discontinuity positions taken
  from the mesh-column averages of the density.

These are the diagnostics CFD-demo's verification tests compute with NumPy
(tests/verification/diagnostics.py, sod_reference.py, ADR 0005 checks); here
they run on device tensors so the 800k-element precision study can use them.
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from .reference_element import DEGREE, build_reference_triangle, vandermonde


# ------------------------------------------------------------ exact solution ---
@dataclass(frozen=True)
class RiemannSide:
    rho: float
    u: float
    p: float


class ExactRiemann:
    """Exact Riemann solution for left/right states (rho, u, p), split at x0."""

    def __init__(self, left, right, gamma: float = 1.4, x0: float = 0.5):
        self.left, self.right = RiemannSide(*left), RiemannSide(*right)
        self.gamma, self.x0 = float(gamma), float(x0)
        self.p_star, self.u_star = self._star()

    def _sound(self, s: RiemannSide) -> float:
        return math.sqrt(self.gamma * s.p / s.rho)

    def _f(self, p: float, s: RiemannSide) -> tuple[float, float]:
        """Velocity change across the wave from side s to pressure p, and its
        derivative in p (shock branch p > p_s, rarefaction branch otherwise)."""
        g = self.gamma
        if p > s.p:
            a = 2.0 / ((g + 1.0) * s.rho)
            b = (g - 1.0) / (g + 1.0) * s.p
            root = math.sqrt(a / (p + b))
            return (p - s.p) * root, root * (1.0 - 0.5 * (p - s.p) / (p + b))
        c = self._sound(s)
        ratio = p / s.p
        e = (g - 1.0) / (2.0 * g)
        return 2.0 * c / (g - 1.0) * (ratio ** e - 1.0), ratio ** (-(g + 1.0) / (2.0 * g)) / (s.rho * c)

    def _star(self) -> tuple[float, float]:
        lt, rt, g = self.left, self.right, self.gamma
        cl, cr = self._sound(lt), self._sound(rt)
        du = rt.u - lt.u
        if 2.0 * (cl + cr) / (g - 1.0) <= du:
            raise ValueError("The Riemann data generate vacuum.")
        # two-rarefaction estimate as the start
        e = (g - 1.0) / (2.0 * g)
        p = ((cl + cr - 0.5 * (g - 1.0) * du) / (cl / lt.p ** e + cr / rt.p ** e)) ** (1.0 / e)
        p = max(p, 1e-12)
        for _ in range(100):
            fl, dl = self._f(p, lt)
            fr, dr = self._f(p, rt)
            step = (fl + fr + du) / (dl + dr)
            p_new = max(p - step, 1e-14 * p)
            if abs(p_new - p) <= 1e-15 * 0.5 * (p_new + p):
                p = p_new
                break
            p = p_new
        fl, _ = self._f(p, lt)
        fr, _ = self._f(p, rt)
        return p, 0.5 * (lt.u + rt.u) + 0.5 * (fr - fl)

    def _side_waves(self, s: RiemannSide, sign: float) -> dict:
        """Speeds of the wave on one side (sign -1 left, +1 right)."""
        g, ps, us = self.gamma, self.p_star, self.u_star
        c = self._sound(s)
        if ps > s.p:  # shock
            speed = s.u + sign * c * math.sqrt((g + 1.0) / (2.0 * g) * ps / s.p + (g - 1.0) / (2.0 * g))
            rho_star = s.rho * ((ps / s.p + (g - 1.0) / (g + 1.0)) / ((g - 1.0) / (g + 1.0) * ps / s.p + 1.0))
            return {"kind": "shock", "speed": speed, "rho_star": rho_star}
        rho_star = s.rho * (ps / s.p) ** (1.0 / g)
        c_star = c * (ps / s.p) ** ((g - 1.0) / (2.0 * g))
        return {"kind": "rarefaction", "head": s.u + sign * c, "tail": us + sign * c_star, "rho_star": rho_star}

    def wave_positions(self, t: float) -> dict:
        """x of every wave front at time t: rarefaction head/tail or shock per
        side, and the contact."""
        out = {}
        for name, s, sign in (("left", self.left, -1.0), ("right", self.right, 1.0)):
            w = self._side_waves(s, sign)
            if w["kind"] == "shock":
                out[f"{name} shock" if name == "left" else "shock"] = self.x0 + w["speed"] * t
            else:
                out[f"{name} head" if name == "right" else "head"] = self.x0 + w["head"] * t
                out[f"{name} tail" if name == "right" else "tail"] = self.x0 + w["tail"] * t
        out["contact"] = self.x0 + self.u_star * t
        return dict(sorted(out.items(), key=lambda kv: kv[1]))

    def sample(self, x, t: float):
        """(rho, u, p) at positions x (NumPy array or torch tensor) and time t > 0."""
        xp = _namespace(x)
        g = self.gamma
        xi = (x - self.x0) / t
        rho = xp.zeros_like(xi)
        u = xp.zeros_like(xi)
        p = xp.zeros_like(xi)
        for s, sign, side in ((self.left, -1.0, xi <= self.u_star), (self.right, 1.0, xi > self.u_star)):
            w = self._side_waves(s, sign)
            if w["kind"] == "shock":
                outside = (xi < w["speed"]) if sign < 0 else (xi > w["speed"])
                rho = xp.where(side & outside, s.rho, xp.where(side, w["rho_star"], rho))
                u = xp.where(side & outside, s.u, xp.where(side, self.u_star, u))
                p = xp.where(side & outside, s.p, xp.where(side, self.p_star, p))
            else:
                c = self._sound(s)
                head, tail = w["head"], w["tail"]
                outside = (xi < head) if sign < 0 else (xi > head)
                star = (xi > tail) if sign < 0 else (xi < tail)
                # inside the fan: c / c_s = 2/(g+1) - sign (g-1)/((g+1) c_s) (u_s - xi)
                ratio = 2.0 / (g + 1.0) - sign * (g - 1.0) / ((g + 1.0) * c) * (s.u - xi)
                ratio = xp.where(ratio > 0.0, ratio, xp.zeros_like(ratio))
                fan_u = 2.0 / (g + 1.0) * (-sign * c + 0.5 * (g - 1.0) * s.u + xi)
                fan_rho = s.rho * ratio ** (2.0 / (g - 1.0))
                fan_p = s.p * ratio ** (2.0 * g / (g - 1.0))
                rho = xp.where(side & outside, s.rho, xp.where(side & star, w["rho_star"], xp.where(side, fan_rho, rho)))
                u = xp.where(side & outside, s.u, xp.where(side & star, self.u_star, xp.where(side, fan_u, u)))
                p = xp.where(side & outside, s.p, xp.where(side & star, self.p_star, xp.where(side, fan_p, p)))
        return rho, u, p


def _namespace(x):
    try:
        import torch

        if isinstance(x, torch.Tensor):
            return torch
    except ImportError:  # pragma: no cover
        pass
    return np


# --------------------------------------------------------------- quadrature ---
def collapsed_gauss(n: int = 10) -> tuple[np.ndarray, np.ndarray]:
    """Barycentric points (m, 3) and weights (m,) summing to 1 on a triangle:
    an n x n Gauss-Legendre rule on the square mapped by the Duffy collapse."""
    t, w = np.polynomial.legendre.leggauss(n)
    a, b = np.meshgrid(0.5 * (t + 1.0), 0.5 * (t + 1.0), indexing="ij")  # on [0, 1]^2
    wa, wb = np.meshgrid(0.5 * w, 0.5 * w, indexing="ij")
    # (a, b) -> barycentric (l1, l2) = (a (1 - b), b), Jacobian (1 - b); the
    # unit-area triangle has reference area 1/2
    l1, l2 = (a * (1.0 - b)).ravel(), b.ravel()
    weight = (2.0 * wa * wb * (1.0 - b)).ravel()
    return np.stack([1.0 - l1 - l2, l1, l2], axis=-1), weight


def _clip(poly: np.ndarray, x: float, keep_right: bool) -> np.ndarray:
    """Convex polygon clipped to x' >= x (keep_right) or x' <= x."""
    d = (poly[:, 0] - x) if keep_right else (x - poly[:, 0])
    out = []
    n = len(poly)
    for i in range(n):
        j = (i + 1) % n
        if d[i] >= 0.0:
            out.append(poly[i])
        if (d[i] >= 0.0) != (d[j] >= 0.0):
            out.append(poly[i] + d[i] / (d[i] - d[j]) * (poly[j] - poly[i]))
    return np.array(out).reshape(-1, 2)


@dataclass
class Quadrature:
    """Integration points (flattened): physical x, y, weight, parent element,
    reference coordinates r, s. ``uniform`` marks the leading run of points
    that use the same reference points in every unsplit element (m per
    element, elements ``uniform_elements``)."""

    x: np.ndarray
    y: np.ndarray
    weight: np.ndarray
    parent: np.ndarray
    r: np.ndarray
    s: np.ndarray
    points_per_element: int
    uniform_elements: np.ndarray

    @property
    def area(self) -> float:
        return float(self.weight.sum())


def quadrature(mesh, breaks=(), n: int = 10, tol: float = 1e-12) -> Quadrature:
    """Integration points over the mesh; elements crossed by a vertical line
    x = b (b in ``breaks``) are cut along it and fan-triangulated."""
    corners = mesh.vertices[mesh.elements]  # (K, 3, 2)
    bary, w = collapsed_gauss(n)
    breaks = np.sort(np.asarray(breaks, dtype=np.float64).reshape(-1))
    xmin, xmax = corners[..., 0].min(1), corners[..., 0].max(1)
    span = np.maximum(xmax - xmin, tol)
    cut = (breaks[None, :] > (xmin + tol * span)[:, None]) & (breaks[None, :] < (xmax - tol * span)[:, None])
    split = np.flatnonzero(cut.any(1))
    whole = np.setdiff1d(np.arange(len(corners)), split)
    # reference coordinates of the rule's points in the reference triangle (-1,-1), (1,-1), (-1,1)
    ref_r = -bary[:, 0] + bary[:, 1] - bary[:, 2]
    ref_s = -bary[:, 0] - bary[:, 1] + bary[:, 2]
    c = corners[whole]
    area = 0.5 * np.abs((c[:, 1, 0] - c[:, 0, 0]) * (c[:, 2, 1] - c[:, 0, 1])
                        - (c[:, 1, 1] - c[:, 0, 1]) * (c[:, 2, 0] - c[:, 0, 0]))
    phys = np.einsum("qv,kvd->kqd", bary, c)
    xs, ys, ws, ps, rs, ss = [phys[..., 0].ravel()], [phys[..., 1].ravel()], [(area[:, None] * w).ravel()], \
        [np.repeat(whole, len(w))], [np.tile(ref_r, len(whole))], [np.tile(ref_s, len(whole))]
    for e in split:
        edges = np.concatenate(([-np.inf], breaks[cut[e]], [np.inf]))
        tri = corners[e]
        for lo, hi in zip(edges[:-1], edges[1:]):
            piece = tri
            if np.isfinite(lo):
                piece = _clip(piece, lo, keep_right=True)
            if len(piece) >= 3 and np.isfinite(hi):
                piece = _clip(piece, hi, keep_right=False)
            for k in range(1, len(piece) - 1):
                sub = np.stack([piece[0], piece[k], piece[k + 1]])
                a2 = abs((sub[1, 0] - sub[0, 0]) * (sub[2, 1] - sub[0, 1]) - (sub[1, 1] - sub[0, 1]) * (sub[2, 0] - sub[0, 0]))
                if a2 == 0.0:
                    continue
                pts = bary @ sub
                # parent reference coordinates: solve the parent's affine map
                basis = np.stack([tri[1] - tri[0], tri[2] - tri[0]], axis=1)
                lam = np.linalg.solve(basis, (pts - tri[0]).T).T  # (m, 2) barycentric l1, l2
                xs.append(pts[:, 0]); ys.append(pts[:, 1]); ws.append(0.5 * a2 * w)
                ps.append(np.full(len(w), e)); rs.append(2.0 * lam[:, 0] - 1.0); ss.append(2.0 * lam[:, 1] - 1.0)
    cat = np.concatenate
    return Quadrature(cat(xs), cat(ys), cat(ws), cat(ps).astype(np.int64), cat(rs), cat(ss), len(w), whole)


def lagrange_at(r: np.ndarray, s: np.ndarray, reference=None) -> np.ndarray:
    """Values (m, Np) of the nodal Lagrange basis at reference points (r, s)."""
    reference = reference or build_reference_triangle(DEGREE)
    return vandermonde(reference.degree, r, s) @ np.linalg.inv(reference.vandermonde)


def evaluate(q, quad: Quadrature, reference=None):
    """The nodal solution q (Np, K, 4) (torch tensor, any device) at the
    quadrature points: a (M, 4) tensor on q's device."""
    import torch

    reference = reference or build_reference_triangle(DEGREE)
    dev, dt = q.device, q.dtype
    n_uniform = len(quad.uniform_elements) * quad.points_per_element
    m = quad.points_per_element
    interp = torch.as_tensor(lagrange_at(quad.r[:m], quad.s[:m], reference), device=dev, dtype=dt)  # (m, Np)
    whole = torch.as_tensor(quad.uniform_elements, device=dev)
    vals_uniform = torch.einsum("qn,nkc->kqc", interp, q[:, whole, :]).reshape(-1, q.shape[-1])
    if n_uniform == len(quad.x):
        return vals_uniform
    rest = slice(n_uniform, None)
    phi = torch.as_tensor(lagrange_at(quad.r[rest], quad.s[rest], reference), device=dev, dtype=dt)  # (M', Np)
    par = torch.as_tensor(quad.parent[rest], device=dev)
    vals_split = torch.einsum("pn,npc->pc", phi, q[:, par, :])
    return torch.cat([vals_uniform, vals_split])


def primitive(vals, gamma: float):
    rho = vals[..., 0]
    u, v = vals[..., 1] / rho, vals[..., 2] / rho
    return rho, u, v, (gamma - 1.0) * (vals[..., 3] - 0.5 * (vals[..., 1] * u + vals[..., 2] * v))


def l1_errors(q, mesh, exact: ExactRiemann, t: float, gamma: float, n: int = 10) -> dict:
    """Domain-averaged L1 errors of density, pressure, x and y velocity
    against the exact solution, with elements cut at the exact wave positions."""
    import torch

    quad = quadrature(mesh, list(exact.wave_positions(t).values()), n)
    vals = evaluate(q, quad)
    rho, u, v, p = primitive(vals, gamma)
    x = torch.as_tensor(quad.x, device=q.device, dtype=q.dtype)
    w = torch.as_tensor(quad.weight, device=q.device, dtype=q.dtype)
    er, eu, ep = exact.sample(x, t)
    area = quad.area
    l1 = lambda a, b: float((w * (a - b).abs()).sum() / area)  # noqa: E731
    return {"density": l1(rho, er), "pressure": l1(p, ep), "x velocity": l1(u, eu),
            "y velocity": float((w * v.abs()).sum() / area)}


def column_density(q, mesh, nx: int, reference=None):
    """Density averages of the nx mesh columns of a structured rectangle mesh
    (column i holds elements 2 (j nx + i) and 2 (j nx + i) + 1) and the x of
    the faces between neighbouring columns. The element integral of the
    degree-4 nodal density is exact with the nodal cell weights."""
    import torch

    reference = reference or build_reference_triangle(DEGREE)
    w = torch.as_tensor(reference.cell_weights / reference.cell_weights.sum(), device=q.device, dtype=q.dtype)
    avg = torch.einsum("n,nk->k", w, q[..., 0])
    c = mesh.vertices[mesh.elements]
    area = torch.as_tensor(0.5 * np.abs((c[:, 1, 0] - c[:, 0, 0]) * (c[:, 2, 1] - c[:, 0, 1])
                                        - (c[:, 1, 1] - c[:, 0, 1]) * (c[:, 2, 0] - c[:, 0, 0])),
                           device=q.device, dtype=q.dtype)
    col = torch.as_tensor((np.arange(len(c)) // 2) % nx, device=q.device)
    mass = torch.zeros(nx, device=q.device, dtype=q.dtype).index_add_(0, col, area * avg)
    total = torch.zeros(nx, device=q.device, dtype=q.dtype).index_add_(0, col, area)
    lo, hi = mesh.vertices[:, 0].min(), mesh.vertices[:, 0].max()
    return (mass / total).cpu().numpy(), lo + (hi - lo) * np.arange(1, nx) / nx


def front_position(column_avg: np.ndarray, face_x: np.ndarray, window) -> float:
    """The column face with the largest density drop (left minus right)
    inside ``window`` (an interval of x)."""
    inside = (face_x >= window[0]) & (face_x <= window[1])
    if not inside.any():
        raise ValueError(f"No column face lies in {window}.")
    drop = np.where(inside, column_avg[:-1] - column_avg[1:], -np.inf)
    return float(face_x[int(np.argmax(drop))])
