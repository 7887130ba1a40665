"""Degree-4 nodal reference triangle: nodes, operators and limiter tables.

Host-side NumPy, built once. The tables are the same as CFD-demo's
(src/cfd_demo/reference_element.py:264-316): warp-and-blend nodes of
Hesthaven & Warburton (Nodal DG Methods, 2008, sec. 6.1; alpha = 0.1001 for
N = 4, table 6.1), the orthonormal Koornwinder-Dubiner basis, Dr/Ds = Vr/Vs
V^-1, LIFT = V V^T E, integration weights 1^T M, GLL face weights, and the
face-midpoint P1 tables of the troubled-cell limiter. The node ORDER is part
of the interface (states are indexed by it): row by row in s, increasing r.

The CUDA kernels do not read these arrays at run time: ``build.py`` prints
them as compile-time constants into ``csrc/tables.cuh``.
"""

from __future__ import annotations

from dataclasses import dataclass
from math import gamma as _G

import numpy as np

DEGREE = 4
NUM_NODES = 15
NUM_FACE_NODES = 5
_ALPHA_OPT = {4: 0.1001}


def _jacobi_table(x: np.ndarray, a: float, b: float, n: int) -> list[np.ndarray]:
    """Orthonormal Jacobi polynomials P_0..P_n^(a,b) at x (three-term recurrence)."""
    x = np.asarray(x, dtype=np.float64)
    g0 = 2.0 ** (a + b + 1) / (a + b + 1) * _G(a + 1) * _G(b + 1) / _G(a + b + 1)
    out = [np.full_like(x, 1.0 / np.sqrt(g0))]
    if n == 0:
        return out
    g1 = (a + 1) * (b + 1) / (a + b + 3) * g0
    out.append(((a + b + 2) * x / 2 + (a - b) / 2) / np.sqrt(g1))
    ap = 2 / (2 + a + b) * np.sqrt((a + 1) * (b + 1) / (a + b + 3))
    for i in range(1, n):
        h = 2 * i + a + b
        an = 2 / (h + 2) * np.sqrt((i + 1) * (i + 1 + a + b) * (i + 1 + a) * (i + 1 + b) / (h + 1) / (h + 3))
        bn = -(a * a - b * b) / h / (h + 2)
        out.append((-ap * out[-2] + (x - bn) * out[-1]) / an)
        ap = an
    return out


def _p(x, a, b, n):
    return _jacobi_table(x, a, b, n)[n]


def _dp(x, a, b, n):
    if n == 0:
        return np.zeros_like(np.asarray(x, dtype=np.float64))
    return np.sqrt(n * (n + a + b + 1)) * _p(x, a + 1, b + 1, n - 1)


def gll_points(n: int) -> np.ndarray:
    """Gauss-Lobatto-Legendre points: +-1 and the Gauss-Jacobi(1,1) points,
    the eigenvalues of the symmetric Jacobi matrix (Golub-Welsch). The matrix
    is formed and diagonalised (LAPACK syevd with vectors) exactly as CFD-demo
    does (reference_element.py:65-93), so the nodes agree to the last bit."""
    if n == 1:
        return np.array([-1.0, 1.0])
    m, a, b = n - 2, 1.0, 1.0
    h1 = 2.0 * np.arange(m + 1) + a + b
    k = np.arange(1, m + 1, dtype=np.float64)
    diag = -0.5 * (a * a - b * b) / (h1 + 2) / h1
    diag[0] = 0.0
    off = 2 / (h1[:m] + 2) * np.sqrt(k * (k + a + b) * (k + a) * (k + b) / (h1[:m] + 1) / (h1[:m] + 3))
    inner, _ = np.linalg.eigh(np.diag(diag) + np.diag(off, 1) + np.diag(off, -1))
    return np.concatenate(([-1.0], inner, [1.0]))


def _warp(n: int, r: np.ndarray) -> np.ndarray:
    """Edge warp (GLL minus equispaced, interpolated) divided by the blend."""
    req = np.linspace(-1.0, 1.0, n + 1)
    v_eq = np.stack(_jacobi_table(req, 0.0, 0.0, n), axis=-1)
    p_r = np.stack(_jacobi_table(r, 0.0, 0.0, n))
    w = np.linalg.solve(v_eq.T, p_r).T @ (gll_points(n) - req)
    inside = (np.abs(r) < 1.0 - 1.0e-10).astype(np.float64)
    return w / (1.0 - (inside * r) ** 2) + w * (inside - 1.0)


def nodes(n: int = DEGREE) -> tuple[np.ndarray, np.ndarray]:
    """Warp-and-blend nodes (r, s) of the reference triangle (-1,-1),(1,-1),(-1,1)."""
    alpha = _ALPHA_OPT.get(n, 0.0)
    lat = [(i / n, m / n) for i in range(n + 1) for m in range(n + 1 - i)]
    b1 = np.array([p[0] for p in lat])
    b3 = np.array([p[1] for p in lat])
    b2 = 1.0 - b1 - b3
    x = -b2 + b3
    y = (-b2 - b3 + 2 * b1) / np.sqrt(3.0)
    w1 = 4 * b2 * b3 * _warp(n, b3 - b2) * (1 + (alpha * b1) ** 2)
    w2 = 4 * b1 * b3 * _warp(n, b1 - b3) * (1 + (alpha * b2) ** 2)
    w3 = 4 * b1 * b2 * _warp(n, b2 - b1) * (1 + (alpha * b3) ** 2)
    x = x + w1 + np.cos(2 * np.pi / 3) * w2 + np.cos(4 * np.pi / 3) * w3
    y = y + np.sin(2 * np.pi / 3) * w2 + np.sin(4 * np.pi / 3) * w3
    l1 = (np.sqrt(3.0) * y + 1.0) / 3.0
    l2 = (-3.0 * x - np.sqrt(3.0) * y + 2.0) / 6.0
    l3 = (3.0 * x - np.sqrt(3.0) * y + 2.0) / 6.0
    return -l2 + l3 - l1, -l2 - l3 + l1


def _basis_modes(n: int):
    return [(i, j) for i in range(n + 1) for j in range(n + 1 - i)]


def _ab(r, s):
    top = np.abs(1.0 - s) < 1e-12
    return np.where(top, -1.0, 2.0 * (1.0 + r) / np.where(top, 1.0, 1.0 - s) - 1.0), s


def vandermonde(n: int, r, s) -> np.ndarray:
    a, b = _ab(np.asarray(r, float), np.asarray(s, float))
    return np.stack([np.sqrt(2.0) * _p(a, 0, 0, i) * _p(b, 2 * i + 1.0, 0, j) * (1 - b) ** i
                     for i, j in _basis_modes(n)], axis=-1)


def grad_vandermonde(n: int, r, s):
    a, b = _ab(np.asarray(r, float), np.asarray(s, float))
    cols_r, cols_s = [], []
    for i, j in _basis_modes(n):
        fa, dfa = _p(a, 0, 0, i), _dp(a, 0, 0, i)
        gb, dgb = _p(b, 2 * i + 1.0, 0, j), _dp(b, 2 * i + 1.0, 0, j)
        hb = 0.5 * (1 - b)
        dr = dfa * gb
        ds = dfa * (gb * (0.5 * (1 + a)))
        if i > 0:
            dr = dr * hb ** (i - 1)
            ds = ds * hb ** (i - 1)
        t = dgb * hb**i
        if i > 0:
            t = t - 0.5 * i * gb * hb ** (i - 1)
        ds = ds + fa * t
        cols_r.append(2.0 ** (i + 0.5) * dr)
        cols_s.append(2.0 ** (i + 0.5) * ds)
    return np.stack(cols_r, axis=-1), np.stack(cols_s, axis=-1)


@dataclass(frozen=True, eq=False)
class ReferenceTriangle:
    """Tables of the degree-4 nodal triangle (same fields as CFD-demo's
    ReferenceTriangle, reference_element.py:213-261)."""

    degree: int
    r: np.ndarray
    s: np.ndarray
    vandermonde: np.ndarray
    mass: np.ndarray
    dr: np.ndarray
    ds: np.ndarray
    face_nodes: np.ndarray  # (3, 5): face 0 = s=-1, 1 = r+s=0, 2 = r=-1
    lift: np.ndarray  # (15, 15) for face data ordered face_nodes.ravel()
    cell_weights: np.ndarray  # (15,) sums to 2
    face_weights: np.ndarray  # (3, 5) GLL weights
    face_midpoint_nodes: np.ndarray  # (3,)
    p1_midpoint: np.ndarray  # (3, 15)
    linear_midpoint_basis: np.ndarray  # (15, 3)

    @property
    def num_nodes(self) -> int:
        return self.r.size

    @property
    def num_face_nodes(self) -> int:
        return self.face_nodes.shape[1]


def build_reference_triangle(n: int = DEGREE) -> ReferenceTriangle:
    if n != DEGREE:
        raise ValueError("The B200 kernels are compiled for degree 4 only.")
    r, s = nodes(n)
    V = vandermonde(n, r, s)
    Vi = np.linalg.inv(V)
    Vr, Vs = grad_vandermonde(n, r, s)
    on_face = (np.abs(s + 1) < 1e-10, np.abs(r + s) < 1e-10, np.abs(r + 1) < 1e-10)
    fn = np.stack([np.flatnonzero(m) for m in on_face])
    nfp = n + 1
    E = np.zeros((r.size, 3 * nfp))
    fw = np.zeros((3, nfp))
    for f, t in enumerate((r[fn[0]], r[fn[1]], s[fn[2]])):
        V1 = np.stack(_jacobi_table(t, 0.0, 0.0, n), axis=-1)
        M1 = np.linalg.inv(V1 @ V1.T)
        E[fn[f], f * nfp:(f + 1) * nfp] = M1
        fw[f] = M1.sum(axis=1)
    mass = Vi.T @ Vi
    mids = fn[:, n // 2]
    lin = [k for k, (i, j) in enumerate(_basis_modes(n)) if i + j <= 1]
    return ReferenceTriangle(
        degree=n, r=r, s=s, vandermonde=V, mass=mass, dr=Vr @ Vi, ds=Vs @ Vi, face_nodes=fn,
        lift=V @ (V.T @ E), cell_weights=mass.sum(axis=0), face_weights=fw, face_midpoint_nodes=mids,
        p1_midpoint=(V[:, lin] @ Vi[lin, :])[mids, :], linear_midpoint_basis=np.stack([-s, 1.0 + r + s, -r], axis=-1),
    )
