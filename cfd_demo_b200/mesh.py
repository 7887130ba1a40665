"""Conforming triangle meshes with tagged boundaries (host side, NumPy).

Same interface and conventions as CFD-demo's src/cfd_demo/mesh.py: elements are
counterclockwise, local face f joins local vertices f and f+1 (mod 3), and
element i is the affine image of the reference triangle (-1,-1), (1,-1),
(-1,1) with local vertex v mapped to reference vertex v. Everything here is
vectorised so that a 1M-element mesh is set up in seconds.
"""

from __future__ import annotations

from collections.abc import Mapping
from dataclasses import dataclass
from types import MappingProxyType

import numpy as np

NUM_FACES = 3


def _frozen(a: np.ndarray) -> np.ndarray:
    a = np.array(a, copy=True)
    a.setflags(write=False)
    return a


@dataclass(frozen=True, eq=False)
class TriangleMesh:
    """Immutable conforming mesh of straight-sided triangles (mesh.py:27-63).

    vertices (Nv, 2) float64; elements (K, 3) counterclockwise vertex ids;
    boundary_edges: tag -> (n, 2) vertex-id pairs.
    """

    vertices: np.ndarray
    elements: np.ndarray
    boundary_edges: Mapping[str, np.ndarray]

    def __post_init__(self) -> None:
        v = np.asarray(self.vertices, dtype=np.float64)
        e = np.asarray(self.elements)
        if v.ndim != 2 or v.shape[1] != 2:
            raise ValueError("vertices must have shape (Nv, 2).")
        if e.ndim != 2 or e.shape[1] != 3 or not np.issubdtype(e.dtype, np.integer):
            raise ValueError("elements must be an integer array of shape (K, 3).")
        if e.size and (e.min() < 0 or e.max() >= len(v)):
            raise ValueError("elements reference vertices that do not exist.")
        edges = {str(t): _frozen(np.asarray(p, dtype=np.int64).reshape(-1, 2)) for t, p in self.boundary_edges.items()}
        object.__setattr__(self, "vertices", _frozen(v))
        object.__setattr__(self, "elements", _frozen(e.astype(np.int64)))
        object.__setattr__(self, "boundary_edges", MappingProxyType(edges))
        if np.any(signed_areas(self) <= 0.0):
            raise ValueError("Every element must have counterclockwise vertices and positive area.")

    @property
    def num_elements(self) -> int:
        return self.elements.shape[0]


def signed_areas(mesh: TriangleMesh) -> np.ndarray:
    p0, p1, p2 = (mesh.vertices[mesh.elements[:, i]] for i in range(3))
    return 0.5 * ((p1[:, 0] - p0[:, 0]) * (p2[:, 1] - p0[:, 1]) - (p2[:, 0] - p0[:, 0]) * (p1[:, 1] - p0[:, 1]))


def rectangle_mesh(nx: int, ny: int, x_range=(0.0, 1.0), y_range=(0.0, 1.0)) -> TriangleMesh:
    """nx*ny rectangles, each split along its lower-left -> upper-right diagonal;
    cell (i, j) owns elements 2(j nx + i) (lower-right) and 2(j nx + i)+1
    (upper-left); tags left/right/bottom/top (mesh.py:72-112)."""
    if nx < 1 or ny < 1:
        raise ValueError("nx and ny must be positive.")
    (x0, x1), (y0, y1) = x_range, y_range
    xs = x0 + (x1 - x0) * (np.arange(nx + 1) / nx)
    ys = y0 + (y1 - y0) * (np.arange(ny + 1) / ny)
    vx, vy = np.meshgrid(xs, ys)
    verts = np.stack([vx.ravel(), vy.ravel()], axis=-1)
    ci, cj = (a.ravel() for a in np.meshgrid(np.arange(nx), np.arange(ny)))
    a = cj * (nx + 1) + ci  # lower-left corner of each cell
    elems = np.empty((2 * nx * ny, 3), dtype=np.int64)
    elems[0::2] = np.stack([a, a + 1, a + nx + 2], axis=-1)
    elems[1::2] = np.stack([a, a + nx + 2, a + nx + 1], axis=-1)
    c, r = np.arange(nx), np.arange(ny)
    edges = {
        "bottom": np.stack([c, c + 1], axis=-1),
        "top": np.stack([ny * (nx + 1) + c, ny * (nx + 1) + c + 1], axis=-1),
        "left": np.stack([r * (nx + 1), (r + 1) * (nx + 1)], axis=-1),
        "right": np.stack([r * (nx + 1) + nx, (r + 1) * (nx + 1) + nx], axis=-1),
    }
    return TriangleMesh(vertices=verts, elements=elems, boundary_edges=edges)


def jittered_rectangle_mesh(nx: int, ny: int, amplitude: float, seed: int,
                            x_range=(0.0, 1.0), y_range=(0.0, 1.0)) -> TriangleMesh:
    """rectangle_mesh with every interior vertex moved by seeded uniform
    +-amplitude * h in each direction (h = cell width / height)."""
    m = rectangle_mesh(nx, ny, x_range, y_range)
    v = np.array(m.vertices)
    (x0, x1), (y0, y1) = x_range, y_range
    eps = 1e-12 * max(x1 - x0, y1 - y0)
    inside = (v[:, 0] > x0 + eps) & (v[:, 0] < x1 - eps) & (v[:, 1] > y0 + eps) & (v[:, 1] < y1 - eps)
    d = np.random.default_rng(seed).uniform(-1.0, 1.0, size=v.shape)
    v[inside] += amplitude * d[inside] * np.array([(x1 - x0) / nx, (y1 - y0) / ny])
    return TriangleMesh(vertices=v, elements=m.elements, boundary_edges=m.boundary_edges)


def sheared_rectangle_mesh(nx: int, ny: int, slope_angle: float, x_range=(0.0, 1.0),
                           y_range=(0.0, 1.0)) -> TriangleMesh:
    """rectangle_mesh mapped by (x, y) -> (x, y + x tan(slope_angle)), the
    affine shear of CFD-demo's proposed ADR 0012 (docs/adr/0012-...:22-31):
    vertices only, so the elements, the lower-left to upper-right diagonal
    and the tags are those of the rectangle; `bottom` becomes the inclined
    wall y = x tan(slope_angle) + y0 and `top` the sheared upper boundary.
    slope_angle in radians, |slope_angle| < pi/2; zero gives rectangle_mesh
    exactly."""
    if not abs(slope_angle) < 0.5 * np.pi:
        raise ValueError("slope_angle must lie strictly between -pi/2 and pi/2.")
    m = rectangle_mesh(nx, ny, x_range, y_range)
    if slope_angle == 0.0:
        return m
    v = np.array(m.vertices)
    v[:, 1] = v[:, 1] + v[:, 0] * np.tan(slope_angle)
    return TriangleMesh(vertices=v, elements=m.elements, boundary_edges=m.boundary_edges)


@dataclass(frozen=True, eq=False)
class MeshConnectivity:
    """Face connectivity (mesh.py:115-132): neighbour element / local face per
    face (-1 on the boundary), sorted boundary tags, per-face tag index (-1
    interior)."""

    neighbor_element: np.ndarray
    neighbor_face: np.ndarray
    boundary_tags: tuple
    face_tag: np.ndarray


def _edge_codes(pairs: np.ndarray, nv: int) -> np.ndarray:
    lo = np.minimum(pairs[..., 0], pairs[..., 1])
    hi = np.maximum(pairs[..., 0], pairs[..., 1])
    return lo * np.int64(nv) + hi


def build_connectivity(mesh: TriangleMesh) -> MeshConnectivity:
    """Match faces by their vertex pairs; reject non-conforming meshes and
    untagged or doubly tagged boundary edges (mesh.py:135-185)."""
    k = mesh.num_elements
    nv = len(mesh.vertices)
    ends = np.stack([mesh.elements, np.roll(mesh.elements, -1, axis=1)], axis=-1).reshape(-1, 2)
    code = _edge_codes(ends, nv)
    order = np.argsort(code, kind="stable")
    sc = code[order]
    if sc.size > 2 and np.any(sc[2:] == sc[:-2]):
        raise ValueError("Nonconforming mesh: a face is shared by more than two elements.")
    pair = np.flatnonzero(sc[1:] == sc[:-1])
    nb_e = np.full(3 * k, -1, dtype=np.int64)
    nb_f = np.full(3 * k, -1, dtype=np.int64)
    a, b = order[pair], order[pair + 1]
    nb_e[a], nb_f[a] = b // 3, b % 3
    nb_e[b], nb_f[b] = a // 3, a % 3

    tags = tuple(sorted(mesh.boundary_edges))
    tag_codes = [_edge_codes(mesh.boundary_edges[t], nv) for t in tags]
    all_codes = np.concatenate(tag_codes) if tag_codes else np.zeros(0, np.int64)
    all_tags = np.concatenate([np.full(len(c), i) for i, c in enumerate(tag_codes)]) if tag_codes else np.zeros(0, np.int64)
    uniq, counts = np.unique(all_codes, return_counts=True)
    if np.any(counts > 1):
        bad = uniq[counts > 1][0]
        raise ValueError(f"Boundary edge {(int(bad // nv), int(bad % nv))} has more than one tag.")
    face_tag = np.full(3 * k, -1, dtype=np.int64)
    bfaces = np.flatnonzero(nb_e < 0)
    srt = np.argsort(all_codes)
    sorted_codes = all_codes[srt]
    pos = np.searchsorted(sorted_codes, code[bfaces])
    pos_c = np.minimum(pos, max(len(sorted_codes) - 1, 0))
    found = (pos < len(sorted_codes)) & (sorted_codes[pos_c] == code[bfaces]) if len(sorted_codes) else np.zeros(len(bfaces), bool)
    if not np.all(found):
        f = int(bfaces[np.flatnonzero(~found)[0]])
        key = (int(code[f] // nv), int(code[f] % nv))
        raise ValueError(f"Boundary face {f % 3} of element {f // 3} (vertices {key}) has no tag.")
    face_tag[bfaces] = all_tags[srt][pos_c]
    if len(bfaces) != len(all_codes):
        used = np.zeros(len(all_codes), bool)
        used[srt[pos_c]] = True
        leftover = all_codes[~used][:5]
        raise ValueError(f"Tagged edges are not boundary faces: {[(int(c // nv), int(c % nv)) for c in leftover]}.")
    shape = (k, 3)
    return MeshConnectivity(_frozen(nb_e.reshape(shape)), _frozen(nb_f.reshape(shape)), tags, _frozen(face_tag.reshape(shape)))


@dataclass(frozen=True, eq=False)
class ElementGeometry:
    """Affine geometry (mesh.py:188-213): J = |K|/2, inverse-map derivatives,
    centroids, outward unit normals (K, 3, 2), edge lengths (K, 3), face
    midpoints (K, 3, 2)."""

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
    """Geometric factors from the vertex coordinates, so that both sides of an
    interior face get exactly opposite normals and equal lengths
    (mesh.py:216-243)."""
    c = mesh.vertices[mesh.elements]
    xr, xs = 0.5 * (c[:, 1, 0] - c[:, 0, 0]), 0.5 * (c[:, 2, 0] - c[:, 0, 0])
    yr, ys = 0.5 * (c[:, 1, 1] - c[:, 0, 1]), 0.5 * (c[:, 2, 1] - c[:, 0, 1])
    jac = xr * ys - xs * yr
    nxt = np.roll(c, -1, axis=1)
    dx, dy = nxt[..., 0] - c[..., 0], nxt[..., 1] - c[..., 1]
    length = np.sqrt(dx * dx + dy * dy)
    return ElementGeometry(
        jacobian=_frozen(jac), rx=_frozen(ys / jac), ry=_frozen(-xs / jac), sx=_frozen(-yr / jac), sy=_frozen(xr / jac),
        centroid=_frozen(c.mean(axis=1)), normal=_frozen(np.stack([dy / length, -dx / length], axis=-1)),
        edge_length=_frozen(length), face_midpoint=_frozen(0.5 * (c + nxt)),
    )


def node_coordinates(mesh: TriangleMesh, r: np.ndarray, s: np.ndarray):
    """Physical node coordinates (x, y), each (Np, K) (mesh.py:246-251)."""
    c = mesh.vertices[mesh.elements]
    w = np.stack([-(r + s) / 2, (1 + r) / 2, (1 + s) / 2], axis=-1)
    p = np.einsum("nv,kvd->nkd", w, c)
    return p[..., 0], p[..., 1]
