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
* ``ObliqueShock``: the steady attached oblique shock of a uniform supersonic
  stream turned by a wedge (the theta-beta-M relation, weak branch, and the
  normal-shock jumps; Anderson, "Modern Compressible Flow", ch. 4), the
  exact solution of CFD-demo's proposed ADR 0011 verification case, with
  exact cell averages over triangles; ``oblique_l1_errors`` and
  ``shock_angle_at`` are its diagnostics.

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


def _clip_line(poly: np.ndarray, normal, c: float, keep_above: bool) -> np.ndarray:
    """Convex polygon clipped to n . p >= c (keep_above) or n . p <= c."""
    d = poly @ np.asarray(normal, dtype=np.float64) - c
    if not keep_above:
        d = -d
    out = []
    n = len(poly)
    for i in range(n):
        j = (i + 1) % n
        if d[i] >= 0.0:
            out.append(poly[i])
        if (d[i] >= 0.0) != (d[j] >= 0.0):
            out.append(poly[i] + d[i] / (d[i] - d[j]) * (poly[j] - poly[i]))
    return np.array(out).reshape(-1, 2)


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


def quadrature(mesh, breaks=(), n: int = 10, tol: float = 1e-12, lines=()) -> Quadrature:
    """Integration points over the mesh; elements crossed by a vertical line
    x = b (b in ``breaks``) or by a line n . p = c ((nx, ny, c) in ``lines``,
    n a unit normal) are cut along it and fan-triangulated."""
    corners = mesh.vertices[mesh.elements]  # (K, 3, 2)
    bary, w = collapsed_gauss(n)
    breaks = np.sort(np.asarray(breaks, dtype=np.float64).reshape(-1))
    xmin, xmax = corners[..., 0].min(1), corners[..., 0].max(1)
    span = np.maximum(xmax - xmin, tol)
    cut = (breaks[None, :] > (xmin + tol * span)[:, None]) & (breaks[None, :] < (xmax - tol * span)[:, None])
    lines = [tuple(float(v) for v in ln) for ln in lines]
    line_cut = np.zeros((len(corners), len(lines)), dtype=bool)
    for li, (lnx, lny, lc) in enumerate(lines):
        d = corners[..., 0] * lnx + corners[..., 1] * lny - lc
        line_cut[:, li] = (d.max(1) > tol * span) & (d.min(1) < -tol * span)
    split = np.flatnonzero(cut.any(1) | line_cut.any(1))
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
        slabs = []
        for lo, hi in zip(edges[:-1], edges[1:]):
            piece = tri
            if np.isfinite(lo):
                piece = _clip(piece, lo, keep_right=True)
            if len(piece) >= 3 and np.isfinite(hi):
                piece = _clip(piece, hi, keep_right=False)
            slabs.append(piece)
        for li in np.flatnonzero(line_cut[e]):
            lnx, lny, lc = lines[li]
            slabs = [h for p in slabs if len(p) >= 3
                     for h in (_clip_line(p, (lnx, lny), lc, True), _clip_line(p, (lnx, lny), lc, False))]
        for piece in slabs:
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


# ------------------------------------------------------ oblique shock (ADR 0011) ---
class ObliqueShock:
    """The steady oblique shock of CFD-demo's proposed verification case
    (docs/adr/0011-oblique-shock-verification.md:31-45): the upstream state
    (rho, u, v, p) = (1, M1, 0, 1/gamma) (sound speed 1) turned by a wall of
    slope angle theta through the attached weak shock y = x tan(beta) from the
    corner at the origin. Below the shock (between it and the wall) the
    post-shock state is uniform and moves parallel to the wall.

    beta solves the theta-beta-M relation
        tan(theta) = 2 cot(beta) (M1^2 sin^2 beta - 1) / (M1^2 (gamma + cos 2 beta) + 2)
    on its weak branch (between the Mach angle asin(1/M1) and the angle of
    maximum deflection); the post-shock state follows from the normal-shock
    jumps at the normal Mach number M1 sin(beta). Only 0 < theta < theta_max(M1)
    is accepted."""

    def __init__(self, mach: float, wall_angle: float, gamma: float = 1.4):
        mach, theta, gamma = float(mach), float(wall_angle), float(gamma)
        if not mach > 1.0:
            raise ValueError("The inflow Mach number must exceed 1.")
        theta_max, beta_max = self.max_deflection(mach, gamma)
        if not 0.0 < theta < theta_max:
            raise ValueError(f"The wall angle must lie in (0, {math.degrees(theta_max):.6f} deg) for an attached "
                             f"shock at Mach {mach}; got {math.degrees(theta):.6f} deg.")
        self.mach, self.theta, self.gamma = mach, theta, gamma
        self.theta_max, self.beta_max = theta_max, beta_max
        lo, hi = math.asin(1.0 / mach), beta_max
        for _ in range(200):  # theta(beta) increases on the weak branch
            mid = 0.5 * (lo + hi)
            if self.deflection(mach, mid, gamma) < theta:
                lo = mid
            else:
                hi = mid
            if hi - lo < 1e-16:
                break
        self.beta = 0.5 * (lo + hi)
        g = gamma
        self.upstream = (1.0, mach, 0.0, 1.0 / g)
        mn1 = mach * math.sin(self.beta)
        rho2 = (g + 1.0) * mn1 * mn1 / ((g - 1.0) * mn1 * mn1 + 2.0)
        p2 = (1.0 + 2.0 * g / (g + 1.0) * (mn1 * mn1 - 1.0)) / g
        mn2 = math.sqrt((1.0 + 0.5 * (g - 1.0) * mn1 * mn1) / (g * mn1 * mn1 - 0.5 * (g - 1.0)))
        m2 = mn2 / math.sin(self.beta - theta)
        speed = m2 * math.sqrt(g * p2 / rho2)
        self.downstream = (rho2, speed * math.cos(theta), speed * math.sin(theta), p2)
        self.downstream_mach = m2

    @staticmethod
    def deflection(mach: float, beta: float, gamma: float = 1.4) -> float:
        """theta(beta) of the theta-beta-M relation."""
        num = 2.0 / math.tan(beta) * (mach * mach * math.sin(beta) ** 2 - 1.0)
        den = mach * mach * (gamma + math.cos(2.0 * beta)) + 2.0
        return math.atan(num / den)

    @classmethod
    def max_deflection(cls, mach: float, gamma: float = 1.4) -> tuple[float, float]:
        """(theta_max, beta at theta_max) by golden-section search: theta(beta)
        is unimodal between the Mach angle and pi/2."""
        a, b = math.asin(1.0 / mach), 0.5 * math.pi
        r = 0.5 * (math.sqrt(5.0) - 1.0)
        c, d = b - r * (b - a), a + r * (b - a)
        fc, fd = cls.deflection(mach, c, gamma), cls.deflection(mach, d, gamma)
        for _ in range(200):
            if fc > fd:
                b, d, fd = d, c, fc
                c = b - r * (b - a)
                fc = cls.deflection(mach, c, gamma)
            else:
                a, c, fc = c, d, fd
                d = a + r * (b - a)
                fd = cls.deflection(mach, d, gamma)
            if b - a < 1e-15:
                break
        beta = 0.5 * (a + b)
        return cls.deflection(mach, beta, gamma), beta

    def _conserved(self, prim) -> np.ndarray:
        rho, u, v, p = prim
        return np.array([rho, rho * u, rho * v, p / (self.gamma - 1.0) + 0.5 * rho * (u * u + v * v)])

    def below_shock(self, x, y):
        """True in the post-shock region: downstream of the corner and below
        the shock line."""
        x, y = np.asarray(x, dtype=np.float64), np.asarray(y, dtype=np.float64)
        return (x > 0.0) & (y < x * math.tan(self.beta))

    def primitive(self, x, y):
        """(rho, u, v, p) arrays of the exact solution at (x, y)."""
        below = self.below_shock(x, y)
        return tuple(np.where(below, d, u_) for u_, d in zip(self.upstream, self.downstream))

    def conserved(self, x, y) -> np.ndarray:
        """Conserved states, shape x.shape + (4,)."""
        below = self.below_shock(x, y)[..., None]
        return np.where(below, self._conserved(self.downstream), self._conserved(self.upstream))

    def cell_average(self, corners: np.ndarray) -> np.ndarray:
        """Exact cell averages (n, 4) over triangles (n, 3, 2): the area of
        each triangle below the shock line (and right of the corner) from
        exact polygon clipping."""
        corners = np.asarray(corners, dtype=np.float64)
        nb = np.array([math.sin(self.beta), -math.cos(self.beta)])  # n . p > 0 below the line
        down, up = self._conserved(self.downstream), self._conserved(self.upstream)
        out = np.empty((len(corners), 4))
        for i, tri in enumerate(corners):
            area = 0.5 * abs((tri[1, 0] - tri[0, 0]) * (tri[2, 1] - tri[0, 1])
                             - (tri[1, 1] - tri[0, 1]) * (tri[2, 0] - tri[0, 0]))
            piece = _clip_line(tri, nb, 0.0, True)
            if len(piece) >= 3:
                piece = _clip_line(piece, (1.0, 0.0), 0.0, True)
            below = 0.0
            for k in range(1, len(piece) - 1):
                a, b, c = piece[0], piece[k], piece[k + 1]
                below += 0.5 * abs((b[0] - a[0]) * (c[1] - a[1]) - (b[1] - a[1]) * (c[0] - a[0]))
            f = min(max(below / area, 0.0), 1.0)
            out[i] = f * down + (1.0 - f) * up
        return out

    def shock_line(self) -> tuple[float, float, float]:
        """(nx, ny, c) of the shock line n . p = c (unit normal)."""
        return (math.sin(self.beta), -math.cos(self.beta), 0.0)


def oblique_l1_errors(q, mesh, exact: ObliqueShock, gamma: float, n: int = 10, region=None) -> dict:
    """Domain-averaged L1 errors of density, pressure and both velocity
    components against the exact oblique-shock solution, elements cut along
    the shock line. ``region(x, y)`` (a boolean mask function) restricts the
    integral, e.g. to the post-shock region."""
    import torch

    quad = quadrature(mesh, (), n, lines=[exact.shock_line()])
    vals = evaluate(q, quad)
    rho, u, v, p = primitive(vals, gamma)
    keep = np.ones(len(quad.x), dtype=bool) if region is None else np.asarray(region(quad.x, quad.y), dtype=bool)
    w = torch.as_tensor(np.where(keep, quad.weight, 0.0), device=q.device, dtype=q.dtype)
    ex = [torch.as_tensor(a, device=q.device, dtype=q.dtype) for a in exact.primitive(quad.x, quad.y)]
    area = float(w.sum())
    l1 = lambda a, b: float((w * (a - b).abs()).sum() / area)  # noqa: E731
    return {"density": l1(rho, ex[0]), "x velocity": l1(u, ex[1]), "y velocity": l1(v, ex[2]),
            "pressure": l1(p, ex[3]), "area": area}


def point_values(q, mesh, x: np.ndarray, y: np.ndarray, reference=None) -> np.ndarray:
    """The nodal solution q (Np, K, 4) at physical points (x, y) (host
    arrays): each point is located by its barycentric coordinates in the
    elements (brute force, in chunks); returns a (m, 4) host array."""
    import torch

    reference = reference or build_reference_triangle(DEGREE)
    c = mesh.vertices[mesh.elements]  # (K, 3, 2)
    p0, e1, e2 = c[:, 0], c[:, 1] - c[:, 0], c[:, 2] - c[:, 0]
    det = e1[:, 0] * e2[:, 1] - e1[:, 1] * e2[:, 0]
    pts = np.stack([np.asarray(x, dtype=np.float64), np.asarray(y, dtype=np.float64)], axis=-1)
    parent = np.full(len(pts), -1, dtype=np.int64)
    lam = np.zeros((len(pts), 2))
    for s0 in range(0, len(pts), 256):
        d = pts[s0:s0 + 256, None, :] - p0[None]
        l1 = (d[..., 0] * e2[None, :, 1] - d[..., 1] * e2[None, :, 0]) / det[None]
        l2 = (e1[None, :, 0] * d[..., 1] - e1[None, :, 1] * d[..., 0]) / det[None]
        inside = (l1 >= -1e-12) & (l2 >= -1e-12) & (l1 + l2 <= 1.0 + 1e-12)
        first = np.argmax(inside, axis=1)
        ok = inside[np.arange(len(first)), first]
        parent[s0:s0 + 256] = np.where(ok, first, -1)
        lam[s0:s0 + 256, 0] = l1[np.arange(len(first)), first]
        lam[s0:s0 + 256, 1] = l2[np.arange(len(first)), first]
    if (parent < 0).any():
        raise ValueError("A sample point lies outside the mesh.")
    phi = torch.as_tensor(lagrange_at(2.0 * lam[:, 0] - 1.0, 2.0 * lam[:, 1] - 1.0, reference), device=q.device,
                          dtype=q.dtype)
    par = torch.as_tensor(parent, device=q.device)
    return torch.einsum("pn,npc->pc", phi, q[:, par, :]).cpu().numpy()


def shock_angle_at(q, mesh, exact: ObliqueShock, x: float, height: float, samples: int = 2000,
                   reference=None) -> float:
    """The shock angle atan(y_s / x) from the largest density drop (upwards)
    along the vertical cut at x between the wall and the top of the domain
    (wall at y = x tan(theta), top at y = x tan(theta) + height), in radians."""
    y0 = x * math.tan(exact.theta)
    ys = y0 + height * (np.arange(samples) + 0.5) / samples
    rho = point_values(q, mesh, np.full(samples, x), ys, reference)[:, 0]
    i = int(np.argmax(rho[:-1] - rho[1:]))
    return math.atan(0.5 * (ys[i] + ys[i + 1]) / x)
