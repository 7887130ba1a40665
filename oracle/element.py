"""Oracle: the degree-4 nodal reference triangle (test infrastructure only).

Restates ``src/cfd_demo/reference_element.py`` of CFD-demo: warp-and-blend
nodes (Hesthaven & Warburton, Nodal DG Methods, 2008, sec. 6.1, alpha from
table 6.1), the orthonormal Koornwinder-Dubiner Vandermonde matrix, the nodal
differentiation and lift matrices, the integration weights, and the
face-midpoint tables used by the troubled-cell limiter.
"""

from __future__ import annotations

from dataclasses import dataclass
from math import gamma as _gamma_fn

import numpy as np

DEGREE = 4
# reference_element.py:23-26 — optimised warp-and-blend alpha for N = 4.
WARP_ALPHA_N4 = 0.1001


def jacobi(x, a: float, b: float, n: int) -> np.ndarray:
    """Orthonormal Jacobi polynomial P_n^(a,b)(x) by the three-term recurrence
    (reference_element.py:29-54)."""
    x = np.asarray(x, dtype=np.float64)
    g0 = 2.0 ** (a + b + 1) / (a + b + 1) * _gamma_fn(a + 1) * _gamma_fn(b + 1) / _gamma_fn(a + b + 1)
    values = [np.full_like(x, 1.0 / np.sqrt(g0))]
    if n == 0:
        return values[0]
    g1 = (a + 1) * (b + 1) / (a + b + 3) * g0
    values.append(((a + b + 2) * x / 2 + (a - b) / 2) / np.sqrt(g1))
    a_prev = 2 / (2 + a + b) * np.sqrt((a + 1) * (b + 1) / (a + b + 3))
    for i in range(1, n):
        h = 2 * i + a + b
        a_next = 2 / (h + 2) * np.sqrt((i + 1) * (i + 1 + a + b) * (i + 1 + a) * (i + 1 + b) / (h + 1) / (h + 3))
        b_next = -(a * a - b * b) / h / (h + 2)
        values.append((-a_prev * values[-2] + (x - b_next) * values[-1]) / a_next)
        a_prev = a_next
    return values[n]


def jacobi_derivative(x, a: float, b: float, n: int) -> np.ndarray:
    """d/dx of the orthonormal Jacobi polynomial (reference_element.py:57-62)."""
    x = np.asarray(x, dtype=np.float64)
    if n == 0:
        return np.zeros_like(x)
    return np.sqrt(n * (n + a + b + 1)) * jacobi(x, a + 1, b + 1, n - 1)


def gauss_lobatto(n: int) -> np.ndarray:
    """The n+1 Gauss-Lobatto-Legendre points, ascending
    (reference_element.py:65-93): interior points are the Gauss-Jacobi(1,1)
    points from the eigen-decomposition (with vectors) of the Jacobi matrix."""
    if n == 1:
        return np.array([-1.0, 1.0])
    m, a, b = n - 2, 1.0, 1.0
    h1 = 2.0 * np.arange(m + 1) + a + b
    k = np.arange(1, m + 1, dtype=np.float64)
    diag = -0.5 * (a * a - b * b) / (h1 + 2) / h1
    diag[0] = 0.0
    off = 2 / (h1[:m] + 2) * np.sqrt(k * (k + a + b) * (k + a) * (k + b) / (h1[:m] + 1) / (h1[:m] + 3))
    interior, _ = np.linalg.eigh(np.diag(diag) + np.diag(off, 1) + np.diag(off, -1))
    return np.concatenate(([-1.0], interior, [1.0]))


def legendre_vandermonde(n: int, x) -> np.ndarray:
    x = np.asarray(x, dtype=np.float64)
    return np.stack([jacobi(x, 0.0, 0.0, j) for j in range(n + 1)], axis=-1)


def _edge_warp(n: int, r: np.ndarray) -> np.ndarray:
    """1D warp equispaced -> GLL divided by the blend (reference_element.py:102-113)."""
    gll = gauss_lobatto(n)
    req = np.linspace(-1.0, 1.0, n + 1)
    veq = legendre_vandermonde(n, req)
    pm = np.stack([jacobi(r, 0.0, 0.0, i) for i in range(n + 1)])
    lagrange = np.linalg.solve(veq.T, pm)
    warp = lagrange.T @ (gll - req)
    inside = (np.abs(r) < 1.0 - 1.0e-10).astype(np.float64)
    return warp / (1.0 - (inside * r) ** 2) + warp * (inside - 1.0)


def warp_blend_nodes(n: int = DEGREE) -> tuple[np.ndarray, np.ndarray]:
    """Warp-and-blend nodes, row by row in s, increasing r within a row
    (reference_element.py:124-149)."""
    alpha = WARP_ALPHA_N4 if n == 4 else 0.0
    l1 = np.array([i / n for i in range(n + 1) for _ in range(n + 1 - i)])
    l3 = np.array([m / n for i in range(n + 1) for m in range(n + 1 - i)])
    l2 = 1.0 - l1 - l3
    x = -l2 + l3
    y = (-l2 - l3 + 2 * l1) / np.sqrt(3.0)
    w1 = 4 * l2 * l3 * _edge_warp(n, l3 - l2) * (1 + (alpha * l1) ** 2)
    w2 = 4 * l1 * l3 * _edge_warp(n, l1 - l3) * (1 + (alpha * l2) ** 2)
    w3 = 4 * l1 * l2 * _edge_warp(n, l2 - l1) * (1 + (alpha * l3) ** 2)
    x = x + w1 + np.cos(2 * np.pi / 3) * w2 + np.cos(4 * np.pi / 3) * w3
    y = y + np.sin(2 * np.pi / 3) * w2 + np.sin(4 * np.pi / 3) * w3
    # equilateral -> reference (reference_element.py:116-121)
    b1 = (np.sqrt(3.0) * y + 1.0) / 3.0
    b2 = (-3.0 * x - np.sqrt(3.0) * y + 2.0) / 6.0
    b3 = (3.0 * x - np.sqrt(3.0) * y + 2.0) / 6.0
    return -b2 + b3 - b1, -b2 - b3 + b1


def _collapse(r, s):
    """(r, s) -> collapsed (a, b) (reference_element.py:159-166)."""
    top = np.abs(1.0 - s) < 1e-12
    a = np.where(top, -1.0, 2.0 * (1.0 + r) / np.where(top, 1.0, 1.0 - s) - 1.0)
    return a, s


def modes(n: int = DEGREE) -> list[tuple[int, int]]:
    return [(i, j) for i in range(n + 1) for j in range(n + 1 - i)]


def vandermonde(n: int, r, s) -> np.ndarray:
    """Orthonormal simplex basis at (r, s) (reference_element.py:174-200)."""
    a, b = _collapse(np.asarray(r, float), np.asarray(s, float))
    cols = [np.sqrt(2.0) * jacobi(a, 0, 0, i) * jacobi(b, 2 * i + 1.0, 0, j) * (1 - b) ** i for i, j in modes(n)]
    return np.stack(cols, axis=-1)


def grad_vandermonde(n: int, r, s) -> tuple[np.ndarray, np.ndarray]:
    """(d/dr, d/ds) of the orthonormal basis (reference_element.py:178-210)."""
    a, b = _collapse(np.asarray(r, float), np.asarray(s, float))
    vr, vs = [], []
    for i, j in modes(n):
        fa, dfa = jacobi(a, 0, 0, i), jacobi_derivative(a, 0, 0, i)
        gb, dgb = jacobi(b, 2 * i + 1.0, 0, j), jacobi_derivative(b, 2 * i + 1.0, 0, j)
        hb = 0.5 * (1 - b)
        d_r = dfa * gb
        d_s = dfa * (gb * (0.5 * (1 + a)))
        if i > 0:
            d_r = d_r * hb ** (i - 1)
            d_s = d_s * hb ** (i - 1)
        t = dgb * hb**i
        if i > 0:
            t = t - 0.5 * i * gb * hb ** (i - 1)
        d_s = d_s + fa * t
        scale = 2.0 ** (i + 0.5)
        vr.append(scale * d_r)
        vs.append(scale * d_s)
    return np.stack(vr, axis=-1), np.stack(vs, axis=-1)


@dataclass(frozen=True, eq=False)
class ReferenceTriangle:
    """Tables of the nodal reference triangle (reference_element.py:213-261)."""

    degree: int
    r: np.ndarray
    s: np.ndarray
    vandermonde: np.ndarray
    mass: np.ndarray
    dr: np.ndarray
    ds: np.ndarray
    face_nodes: np.ndarray
    lift: np.ndarray
    cell_weights: np.ndarray
    face_weights: np.ndarray
    face_midpoint_nodes: np.ndarray
    p1_midpoint: np.ndarray
    linear_midpoint_basis: np.ndarray

    @property
    def num_nodes(self) -> int:
        return self.r.size

    @property
    def num_face_nodes(self) -> int:
        return self.face_nodes.shape[1]


def build_reference_triangle(n: int = DEGREE) -> ReferenceTriangle:
    """reference_element.py:264-316."""
    r, s = warp_blend_nodes(n)
    v = vandermonde(n, r, s)
    vinv = np.linalg.inv(v)
    mass = vinv.T @ vinv
    vr, vs = grad_vandermonde(n, r, s)
    dr, ds = vr @ vinv, vs @ vinv
    masks = (np.abs(s + 1) < 1e-10, np.abs(r + s) < 1e-10, np.abs(r + 1) < 1e-10)
    face_nodes = np.stack([np.flatnonzero(m) for m in masks])
    nfp = n + 1
    emat = np.zeros((r.size, 3 * nfp))
    face_weights = np.zeros((3, nfp))
    for f, coord in enumerate((r[face_nodes[0]], r[face_nodes[1]], s[face_nodes[2]])):
        v1 = legendre_vandermonde(n, coord)
        m1 = np.linalg.inv(v1 @ v1.T)
        emat[face_nodes[f], f * nfp:(f + 1) * nfp] = m1
        face_weights[f] = m1.sum(axis=1)
    lift = v @ (v.T @ emat)
    mids = face_nodes[:, n // 2]
    lin = [k for k, (i, j) in enumerate(modes(n)) if i + j <= 1]
    p1 = (v[:, lin] @ vinv[lin, :])[mids, :]
    basis = np.stack([-s, 1.0 + r + s, -r], axis=-1)
    return ReferenceTriangle(
        degree=n, r=r, s=s, vandermonde=v, mass=mass, dr=dr, ds=ds, face_nodes=face_nodes, lift=lift,
        cell_weights=mass.sum(axis=0), face_weights=face_weights, face_midpoint_nodes=mids,
        p1_midpoint=p1, linear_midpoint_basis=basis,
    )
