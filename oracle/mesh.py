"""Oracle: conforming triangle meshes, connectivity and affine geometry
(test infrastructure only).

Restates ``src/cfd_demo/mesh.py`` of CFD-demo. Elements are counterclockwise;
local face f joins local vertices f and f+1 (mod 3).
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass(frozen=True, eq=False)
class TriangleMesh:
    """mesh.py:27-63 (validation reduced to what the oracle needs)."""

    vertices: np.ndarray
    elements: np.ndarray
    boundary_edges: dict

    def __post_init__(self) -> None:
        object.__setattr__(self, "vertices", np.asarray(self.vertices, dtype=np.float64))
        object.__setattr__(self, "elements", np.asarray(self.elements, dtype=np.int64))
        edges = {str(t): np.asarray(p, dtype=np.int64).reshape(-1, 2) for t, p in self.boundary_edges.items()}
        object.__setattr__(self, "boundary_edges", edges)
        p0, p1, p2 = (self.vertices[self.elements[:, i]] for i in range(3))
        area2 = (p1[:, 0] - p0[:, 0]) * (p2[:, 1] - p0[:, 1]) - (p2[:, 0] - p0[:, 0]) * (p1[:, 1] - p0[:, 1])
        if np.any(area2 <= 0.0):
            raise ValueError("Every element must have counterclockwise vertices and positive area.")

    @property
    def num_elements(self) -> int:
        return self.elements.shape[0]


def rectangle_mesh(nx: int, ny: int, x_range=(0.0, 1.0), y_range=(0.0, 1.0)) -> TriangleMesh:
    """nx*ny rectangles split lower-left -> upper-right; cell (i, j) holds
    elements 2(j nx + i) (lower-right) and 2(j nx + i)+1 (upper-left)
    (mesh.py:72-112)."""
    (x0, x1), (y0, y1) = x_range, y_range
    xs = x0 + (x1 - x0) * (np.arange(nx + 1) / nx)
    ys = y0 + (y1 - y0) * (np.arange(ny + 1) / ny)
    gx, gy = np.meshgrid(xs, ys)
    vertices = np.stack([gx.ravel(), gy.ravel()], axis=-1)
    i, j = (a.ravel() for a in np.meshgrid(np.arange(nx), np.arange(ny)))

    def vid(a, b):
        return b * (nx + 1) + a

    lower = np.stack([vid(i, j), vid(i + 1, j), vid(i + 1, j + 1)], axis=-1)
    upper = np.stack([vid(i, j), vid(i + 1, j + 1), vid(i, j + 1)], axis=-1)
    elements = np.stack([lower, upper], axis=1).reshape(-1, 3)
    cols, rows = np.arange(nx), np.arange(ny)
    edges = {
        "bottom": np.stack([vid(cols, 0), vid(cols + 1, 0)], axis=-1),
        "top": np.stack([vid(cols, ny), vid(cols + 1, ny)], axis=-1),
        "left": np.stack([vid(0, rows), vid(0, rows + 1)], axis=-1),
        "right": np.stack([vid(nx, rows), vid(nx, rows + 1)], axis=-1),
    }
    return TriangleMesh(vertices, elements, edges)


@dataclass(frozen=True, eq=False)
class MeshConnectivity:
    """mesh.py:115-132."""

    neighbor_element: np.ndarray  # (K, 3), -1 on the boundary
    neighbor_face: np.ndarray  # (K, 3), -1 on the boundary
    boundary_tags: tuple
    face_tag: np.ndarray  # (K, 3), index into boundary_tags, -1 interior


def build_connectivity(mesh: TriangleMesh) -> MeshConnectivity:
    """Face matching by sorted vertex pairs (mesh.py:135-185)."""
    k = mesh.num_elements
    ends = np.stack([mesh.elements, np.roll(mesh.elements, -1, axis=1)], axis=-1).reshape(-1, 2)
    keys = np.sort(ends, axis=1)
    code = keys[:, 0] * (int(keys.max()) + 1) + keys[:, 1]
    order = np.argsort(code, kind="stable")
    sc = code[order]
    same = np.flatnonzero(sc[1:] == sc[:-1])
    if np.any(sc[2:] == sc[:-2]):
        raise ValueError("Nonconforming mesh: a face is shared by more than two elements.")
    nb_e = -np.ones(3 * k, dtype=np.int64)
    nb_f = -np.ones(3 * k, dtype=np.int64)
    a, b = order[same], order[same + 1]
    nb_e[a], nb_f[a] = b // 3, b % 3
    nb_e[b], nb_f[b] = a // 3, a % 3
    tags = tuple(sorted(mesh.boundary_edges))
    lookup = {}
    for ti, tag in enumerate(tags):
        for u, w in mesh.boundary_edges[tag]:
            lookup[(min(u, w), max(u, w))] = ti
    face_tag = -np.ones(3 * k, dtype=np.int64)
    for face in np.flatnonzero(nb_e < 0):
        key = (int(keys[face, 0]), int(keys[face, 1]))
        if key not in lookup:
            raise ValueError(f"Boundary face {face % 3} of element {face // 3} (vertices {key}) has no tag.")
        face_tag[face] = lookup.pop(key)
    if lookup:
        raise ValueError("Tagged edges are not boundary faces.")
    return MeshConnectivity(nb_e.reshape(k, 3), nb_f.reshape(k, 3), tags, face_tag.reshape(k, 3))


@dataclass(frozen=True, eq=False)
class ElementGeometry:
    """mesh.py:188-213."""

    jacobian: np.ndarray
    rx: np.ndarray
    ry: np.ndarray
    sx: np.ndarray
    sy: np.ndarray
    centroid: np.ndarray
    normal: np.ndarray
    edge_length: np.ndarray
    face_midpoint: np.ndarray

    @property
    def area(self) -> np.ndarray:
        return 2.0 * self.jacobian


def element_geometry(mesh: TriangleMesh) -> ElementGeometry:
    """Affine factors from vertex coordinates (mesh.py:216-243)."""
    c = mesh.vertices[mesh.elements]
    xr, xs = 0.5 * (c[:, 1, 0] - c[:, 0, 0]), 0.5 * (c[:, 2, 0] - c[:, 0, 0])
    yr, ys = 0.5 * (c[:, 1, 1] - c[:, 0, 1]), 0.5 * (c[:, 2, 1] - c[:, 0, 1])
    jac = xr * ys - xs * yr
    end = np.roll(c, -1, axis=1)
    dx, dy = end[..., 0] - c[..., 0], end[..., 1] - c[..., 1]
    length = np.sqrt(dx * dx + dy * dy)
    normal = np.stack([dy / length, -dx / length], axis=-1)
    return ElementGeometry(
        jacobian=jac, rx=ys / jac, ry=-xs / jac, sx=-yr / jac, sy=xr / jac, centroid=c.mean(axis=1),
        normal=normal, edge_length=length, face_midpoint=0.5 * (c + end),
    )


def node_coordinates(mesh: TriangleMesh, r: np.ndarray, s: np.ndarray):
    """Physical node coordinates, each (Np, K) (mesh.py:246-251)."""
    c = mesh.vertices[mesh.elements]
    w = np.stack([-(r + s) / 2, (1 + r) / 2, (1 + s) / 2], axis=-1)
    p = np.einsum("nv,kvd->nkd", w, c)
    return p[..., 0], p[..., 1]


def pair_face_nodes(mesh, conn, x, y, face_nodes, rtol: float = 1e-9) -> np.ndarray:
    """Neighbour node index coinciding with each face node, (3, Nfp, K)
    (mesh.py:254-291)."""
    nf, nfp = face_nodes.shape
    k = mesh.num_elements
    partner = np.broadcast_to(face_nodes[:, :, None], (nf, nfp, k)).copy()
    scale = element_geometry(mesh).edge_length
    for f in range(nf):
        el = np.flatnonzero(conn.neighbor_element[:, f] >= 0)
        if el.size == 0:
            continue
        nb = conn.neighbor_element[el, f]
        cand = face_nodes[conn.neighbor_face[el, f]]  # (n, Nfp)
        own = np.stack([x[face_nodes[f]][:, el], y[face_nodes[f]][:, el]], axis=-1)  # (Nfp, n, 2)
        oth = np.stack([x[cand.T, nb[None, :]], y[cand.T, nb[None, :]]], axis=-1)  # (Nfp, n, 2)
        dist = np.linalg.norm(own[:, None] - oth[None, :], axis=-1)  # (Nfp, Nfp, n)
        best = dist.argmin(axis=1)
        if np.any(np.take_along_axis(dist, best[:, None], axis=1)[:, 0] > rtol * scale[el, f][None]):
            raise ValueError("Neighboring face nodes do not coincide; the mesh is not conforming.")
        partner[f][:, el] = np.take_along_axis(cand.T, best, axis=0)
    return partner


def perturbed_mesh(nx: int, ny: int, amplitude: float = 0.25, seed: int = 0) -> TriangleMesh:
    """Rectangle mesh with seeded uniform jitter of the interior vertices, the
    helper of the reference's tests (tests/unit/test_dg_operator.py:19-27)."""
    mesh = rectangle_mesh(nx, ny)
    v = np.array(mesh.vertices)
    inside = np.all((v > 1e-12) & (v < 1.0 - 1e-12), axis=1)
    rng = np.random.default_rng(seed)
    d = rng.uniform(-1.0, 1.0, size=v.shape)
    v[inside] += amplitude * d[inside] / np.array([nx, ny])
    return TriangleMesh(v, mesh.elements, mesh.boundary_edges)
