"""Device tables of the DG operator and limiter, in the kernels' layout.

Host-side, built once per solver (CFD-demo builds the equivalent arrays in
src/cfd_demo/dg.py:76-116 and src/cfd_demo/limiting.py:51-121, in its own
(3 Nfp, K) face-node layout). Here every table is element-major with a padded
leading dimension ``ld`` so that a warp's loads of one field are contiguous:

    metric     [4][ld]  rx, ry, sx, sy                         float64 (+ float32 copy)
    face_geo   [9][ld]  nx_f, ny_f, sJ_f / J for faces f=0,1,2 float64 (+ float32 copy)
    face_hlen  [3][ld]  half edge lengths (boundary-flux weights)
    dt_geo     [ld]     min_e 2|K| / ((N+1)^2 |e|)             (time_integration.py:32-34)
    jacobian   [ld]     J = |K| / 2
    cs_coef    [6][ld]  Cockburn-Shu alpha_f, beta_f           float64 (+ float32 copy)
    neighbor   [3][ld]  neighbour element, or fixed-state row   int32
    face_info  [ld]     per face 8 bits: kind | nbr face << 2 | partner face << 4
    instance   [ld]     instance id (batched meshes only)       int32
    bc_states  [rows][4] fixed exterior states; per exact-state face 6 rows (its 5
                         face-node states, then its ghost average)  float64

Several meshes ("instances") can be concatenated into one table set; element
and neighbour indices are then global.
"""

from __future__ import annotations

from dataclasses import dataclass, field
from typing import NamedTuple

import numpy as np

from . import _native
from .boundary import EXACT_STATE, FIXED_STATE, SLIP_WALL
from .mesh import MeshConnectivity, TriangleMesh, element_geometry, node_coordinates

COEFFICIENT_TOLERANCE = 1e-12  # limiting.py:31
LD_ALIGN = 64


def padded_ld(k: int) -> int:
    return ((k + LD_ALIGN - 1) // LD_ALIGN) * LD_ALIGN


def resolve_boundary_conditions(connectivity: MeshConnectivity, boundary_conditions) -> tuple[np.ndarray, np.ndarray]:
    """Per-face kinds (K, 3) and fixed states (K, 3, 4) (dg.py:52-73)."""
    tags = set(connectivity.boundary_tags)
    missing = sorted(tags - set(boundary_conditions))
    if missing:
        raise ValueError(f"Boundary tags without a boundary condition: {missing}.")
    unknown = sorted(set(boundary_conditions) - tags)
    if unknown:
        raise ValueError(f"Boundary conditions for tags that are not in the mesh: {unknown}.")
    kind = np.zeros(connectivity.face_tag.shape, dtype=np.int32)
    state = np.zeros(connectivity.face_tag.shape + (4,))
    for ti, tag in enumerate(connectivity.boundary_tags):
        bc = boundary_conditions[tag]
        mask = connectivity.face_tag == ti
        kind[mask] = bc.kind
        if bc.kind == FIXED_STATE:
            state[mask] = bc.state
        elif bc.kind not in (SLIP_WALL, EXACT_STATE):
            raise ValueError(f"Unsupported boundary condition for tag {tag!r}: {bc!r}.")
    return kind, state


def reflected_triangles(mesh: TriangleMesh, elements: np.ndarray, faces: np.ndarray) -> np.ndarray:
    """The corners (n, 3, 2) of each listed element reflected across the line
    of its listed face (local face f joins local vertices f and f+1)."""
    c = mesh.vertices[mesh.elements[elements]]  # (n, 3, 2)
    a = c[np.arange(len(faces)), faces]
    b = c[np.arange(len(faces)), (faces + 1) % 3]
    d = b - a
    nrm = np.stack([d[:, 1], -d[:, 0]], axis=-1) / np.linalg.norm(d, axis=-1, keepdims=True)
    off = np.einsum("nvd,nd->nv", c - a[:, None], nrm)
    return c - 2.0 * off[..., None] * nrm[:, None]


def sampled_cell_average(bc, corners: np.ndarray, subdivisions: int = 32) -> np.ndarray:
    """Cell averages (n, 4) of bc.states over triangles (n, 3, 2): the mean of
    the values at the centroids of the subdivisions**2 equal sub-triangles."""
    m = subdivisions
    i, j = np.meshgrid(np.arange(m), np.arange(m), indexing="ij")
    up = (i + j) < m
    b_up = np.stack([(i + 1 / 3), (j + 1 / 3)], axis=-1)[up] / m
    dn = (i + j) < m - 1
    b_dn = np.stack([(i + 2 / 3), (j + 2 / 3)], axis=-1)[dn] / m
    lam = np.concatenate([b_up, b_dn])  # barycentric weights of corners 1 and 2
    w = np.stack([1.0 - lam[:, 0] - lam[:, 1], lam[:, 0], lam[:, 1]], axis=-1)  # (m^2, 3)
    pts = np.einsum("pv,nvd->npd", w, corners)
    return bc.states(pts[..., 0], pts[..., 1]).mean(axis=1)


@dataclass
class ExactRows:
    """Exterior-state rows of the exact-state faces, face by face in (element,
    face) order: the states at the face's nodes (element face-node order) and
    the ghost average across it."""

    elements: np.ndarray  # (n,)
    faces: np.ndarray  # (n,)
    node_states: np.ndarray  # (n, Nfp, 4)
    ghost: np.ndarray  # (n, 4)


def exact_state_rows(mesh: TriangleMesh, connectivity: MeshConnectivity, reference, kind: np.ndarray,
                     boundary_conditions) -> ExactRows:
    """Evaluate every ExactState boundary condition once: at the face nodes of
    its faces (the interface flux's exterior states) and, as the ghost
    average, over each boundary element reflected across the face (the
    condition's own cell_average(corners) when it has one, else a sampled
    average)."""
    e_idx, f_idx = np.nonzero(kind == EXACT_STATE)
    nfp = reference.face_nodes.shape[1]
    node_states = np.zeros((len(e_idx), nfp, 4))
    ghost = np.zeros((len(e_idx), 4))
    if len(e_idx):
        x, y = node_coordinates(mesh, reference.r, reference.s)
        fn = np.asarray(reference.face_nodes)[f_idx]  # (n, Nfp) node ids
        fx, fy = x[fn, e_idx[:, None]], y[fn, e_idx[:, None]]
        corners = reflected_triangles(mesh, e_idx, f_idx)
        tags = connectivity.face_tag[e_idx, f_idx]
        for ti in np.unique(tags):
            sel = tags == ti
            bc = boundary_conditions[connectivity.boundary_tags[ti]]
            node_states[sel] = bc.states(fx[sel], fy[sel])
            average = getattr(bc, "cell_average", None)
            ghost[sel] = average(corners[sel]) if average is not None else sampled_cell_average(bc, corners[sel])
    return ExactRows(e_idx, f_idx, node_states, ghost)


def neighbor_coefficients(connectivity: MeshConnectivity, geometry) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """Nonnegative Cockburn-Shu coefficients per face, (K, 3) each
    (limiting.py:51-94): m_i - b0 = alpha (b_i - b0) + beta (b_j - b0) with
    the first partner face j in (i+1, i+2) that gives alpha, beta >= -tol;
    boundary neighbours use the centroid reflected across the face."""
    cen, mid, nrm = geometry.centroid, geometry.face_midpoint, geometry.normal
    nb = connectivity.neighbor_element
    off = np.sum((mid - cen[:, None, :]) * nrm, axis=-1, keepdims=True)
    ncen = np.where((nb >= 0)[..., None], cen[np.maximum(nb, 0)], cen[:, None, :] + 2.0 * off * nrm)
    d = ncen - cen[:, None, :]
    t = mid - cen[:, None, :]
    k = cen.shape[0]
    alpha = np.zeros((k, 3))
    beta = np.zeros((k, 3))
    partner = np.full((k, 3), -1, dtype=np.int64)
    for f in range(3):
        for shift in (1, 2):
            o = (f + shift) % 3
            di, dj, tt = d[:, f], d[:, o], t[:, f]
            det = di[:, 0] * dj[:, 1] - di[:, 1] * dj[:, 0]
            safe = np.where(det == 0.0, 1.0, det)
            a = (tt[:, 0] * dj[:, 1] - tt[:, 1] * dj[:, 0]) / safe
            b = (di[:, 0] * tt[:, 1] - di[:, 1] * tt[:, 0]) / safe
            pick = (det != 0.0) & (a >= -COEFFICIENT_TOLERANCE) & (b >= -COEFFICIENT_TOLERANCE) & (partner[:, f] < 0)
            alpha[pick, f] = np.maximum(a[pick], 0.0)
            beta[pick, f] = np.maximum(b[pick], 0.0)
            partner[pick, f] = o
    if np.any(partner < 0):
        e, f = np.argwhere(partner < 0)[0]
        raise ValueError(f"No nonnegative Cockburn-Shu neighbor coefficients for face {f} of element {e}.")
    return alpha, beta, partner


def check_face_pairing(mesh: TriangleMesh, connectivity: MeshConnectivity, reference, relative_tolerance=1e-9,
                       *, geometry=None, device=None) -> None:
    """Check by coordinates that face node k of face f meets node 4-k (or k)
    of the neighbour's face, the rule the kernels use (mesh.py:254-291 pairs
    the nodes by coordinates). With a CUDA ``device`` the check runs there
    (it dominates the host setup of large meshes)."""
    geometry = geometry if geometry is not None else element_geometry(mesh)
    fn = np.asarray(reference.face_nodes)
    nfp = fn.shape[1]
    r, s = reference.r[fn], reference.s[fn]  # (3, Nfp)
    bary = np.stack([-(r + s) / 2, (1 + r) / 2, (1 + s) / 2], axis=-1)  # (3, Nfp, 3)
    nbr, nface = connectivity.neighbor_element, connectivity.neighbor_face
    k = np.arange(nfp)
    if device is not None and str(device).startswith("cuda"):
        import torch

        dev = torch.device(device)
        corners = torch.as_tensor(mesh.vertices[mesh.elements], device=dev)  # (K, 3, 2)
        own = torch.einsum("fkv,evd->efkd", torch.as_tensor(bary, device=dev), corners)  # (K, 3, Nfp, 2)
        nb_t = torch.as_tensor(np.array(nbr), device=dev)  # copies: the tables are read-only
        nf_t = torch.as_tensor(np.array(nface), device=dev)
        e_idx, f_idx = torch.nonzero(nb_t >= 0, as_tuple=True)
        nb_i, nf_i = nb_t[e_idx, f_idx], nf_t[e_idx, f_idx]
        same = (f_idx == 2) != (nf_i == 2)
        kt = torch.arange(nfp, device=dev)
        kk = torch.where(same[:, None], kt[None, :], nfp - 1 - kt[None, :])  # (M, Nfp)
        partner = own[nb_i[:, None], nf_i[:, None], kk]  # (M, Nfp, 2)
        dist = torch.linalg.vector_norm(own[e_idx, f_idx] - partner, dim=-1)
        tol = relative_tolerance * torch.as_tensor(np.array(geometry.edge_length), device=dev)[e_idx, f_idx]
        bad = bool((dist > tol[:, None]).any())
    else:
        corners = mesh.vertices[mesh.elements]
        own = np.einsum("fkv,evd->efkd", bary, corners)
        e_idx, f_idx = np.nonzero(nbr >= 0)
        nb_i, nf_i = nbr[e_idx, f_idx], nface[e_idx, f_idx]
        same = (f_idx == 2) != (nf_i == 2)
        kk = np.where(same[:, None], k[None, :], nfp - 1 - k[None, :])
        partner = own[nb_i[:, None], nf_i[:, None], kk]
        dist = np.hypot(*np.moveaxis(own[e_idx, f_idx] - partner, -1, 0))
        bad = bool(np.any(dist > relative_tolerance * geometry.edge_length[e_idx, f_idx][:, None]))
    if bad:
        raise ValueError("Neighboring face nodes do not coincide; the mesh is not conforming.")


class LimiterOperators(NamedTuple):
    """Host (NumPy) copies of the limiter tables under the reference's field
    names (limiting.py:34-48, built by build_limiter_operators, :97-121); face
    arrays are (3, K). The kernels read the same data from the packed
    CfdMesh tables."""

    average_weights: np.ndarray  # (Np,)
    midpoint_nodes: np.ndarray  # (3,)
    p1_midpoint: np.ndarray  # (3, Np)
    linear_basis: np.ndarray  # (Np, 3)
    neighbor: np.ndarray  # (3, K): neighbour element, or the element itself on boundaries
    neighbor_kind: np.ndarray  # (3, K): 0 interior, SLIP_WALL or FIXED_STATE
    normal_x: np.ndarray  # (3, K)
    normal_y: np.ndarray  # (3, K)
    fixed_state: np.ndarray  # (3, K, 4)
    alpha: np.ndarray  # (3, K)
    beta: np.ndarray  # (3, K)
    partner_face: np.ndarray  # (3, K)


def limiter_operators(connectivity: MeshConnectivity, geometry, reference, kind: np.ndarray,
                      state: np.ndarray) -> LimiterOperators:
    alpha, beta, partner = neighbor_coefficients(connectivity, geometry)
    k = connectivity.neighbor_element.shape[0]
    own = np.broadcast_to(np.arange(k)[:, None], (k, 3))
    nbr = np.where(connectivity.neighbor_element >= 0, connectivity.neighbor_element, own)
    w = reference.cell_weights
    return LimiterOperators(
        average_weights=w / w.sum(), midpoint_nodes=np.asarray(reference.face_midpoint_nodes),
        p1_midpoint=np.asarray(reference.p1_midpoint), linear_basis=np.asarray(reference.linear_midpoint_basis),
        neighbor=nbr.T.copy(), neighbor_kind=np.asarray(kind).T.copy(),
        normal_x=geometry.normal[:, :, 0].T.copy(), normal_y=geometry.normal[:, :, 1].T.copy(),
        fixed_state=np.transpose(state, (1, 0, 2)).copy(), alpha=alpha.T.copy(), beta=beta.T.copy(),
        partner_face=np.asarray(partner).T.copy())


@dataclass
class HostTables:
    """One instance's tables on the host (float64 / int32), before upload."""

    num_elements: int
    metric: np.ndarray  # (4, K)
    face_geo: np.ndarray  # (9, K)
    face_hlen: np.ndarray  # (3, K)
    dt_geo: np.ndarray  # (K,)
    jacobian: np.ndarray  # (K,)
    cs_coef: np.ndarray  # (6, K)
    neighbor: np.ndarray  # (3, K) int32 (local element ids, or local bc rows)
    face_info: np.ndarray  # (K,) int32
    bc_states: np.ndarray  # (rows, 4)
    interior: np.ndarray = field(default=None)  # (3, K) bool


def host_tables(mesh: TriangleMesh, connectivity: MeshConnectivity, geometry, reference, kind: np.ndarray,
                state: np.ndarray, degree: int = 4, device=None, boundary_conditions=None) -> HostTables:
    """One mesh's tables. Exact-state faces (kind EXACT_STATE) need the
    boundary conditions to evaluate their rows."""
    k = mesh.num_elements
    check_face_pairing(mesh, connectivity, reference, geometry=geometry, device=device)
    alpha, beta, partner = neighbor_coefficients(connectivity, geometry)
    # fixed-state rows: one per distinct exterior state
    fixed = kind == FIXED_STATE
    rows, inverse = (np.unique(state[fixed], axis=0, return_inverse=True) if fixed.any()
                     else (np.zeros((0, 4)), np.zeros(0, dtype=np.int64)))
    rows = np.asarray(rows, dtype=np.float64).reshape(-1, 4)
    nbr = np.where(connectivity.neighbor_element >= 0, connectivity.neighbor_element, 0).astype(np.int64)
    nbr[fixed] = inverse.reshape(-1)
    if (kind == EXACT_STATE).any():
        if boundary_conditions is None:
            raise ValueError("Exact-state faces need the boundary conditions to build their rows.")
        ex = exact_state_rows(mesh, connectivity, reference, kind, boundary_conditions)
        nfp = ex.node_states.shape[1]
        blocks = np.concatenate([ex.node_states, ex.ghost[:, None]], axis=1).reshape(-1, 4)  # (n (Nfp+1), 4)
        nbr[ex.elements, ex.faces] = len(rows) + (nfp + 1) * np.arange(len(ex.elements))
        rows = np.concatenate([rows, blocks])
    nface = np.where(connectivity.neighbor_face >= 0, connectivity.neighbor_face, 0)
    info = np.zeros(k, dtype=np.int64)
    for f in range(3):
        field8 = kind[:, f].astype(np.int64) | (nface[:, f] << 2) | (partner[:, f] << 4)
        info |= field8 << (8 * f)
    fscale = 0.5 * geometry.edge_length / geometry.jacobian[:, None]  # dg.py:99
    face_geo = np.empty((9, k))
    for f in range(3):
        face_geo[3 * f] = geometry.normal[:, f, 0]
        face_geo[3 * f + 1] = geometry.normal[:, f, 1]
        face_geo[3 * f + 2] = fscale[:, f]
    dt_geo = np.min(2.0 * geometry.area[:, None] / ((degree + 1) ** 2 * geometry.edge_length), axis=1)
    return HostTables(
        num_elements=k,
        metric=np.stack([geometry.rx, geometry.ry, geometry.sx, geometry.sy]),
        face_geo=face_geo,
        face_hlen=(0.5 * geometry.edge_length).T.copy(),
        dt_geo=dt_geo,
        jacobian=np.asarray(geometry.jacobian, dtype=np.float64),
        cs_coef=np.concatenate([alpha.T, beta.T]),
        neighbor=nbr.T.astype(np.int32),
        face_info=info.astype(np.int32),
        bc_states=rows,
        interior=(connectivity.neighbor_element >= 0).T,
    )


def boundary_tag_tables(mesh: TriangleMesh, boundary_conditions) -> tuple[list, np.ndarray, np.ndarray, np.ndarray]:
    """Per tag (sorted names, as mesh.py:150 orders them): boundary kind and
    fixed-state row, and the distinct fixed exterior states (rows sorted as
    np.unique sorts them, the host builder's bc_states). Raises the host
    builder's errors for missing or unknown tags."""
    tags = sorted(mesh.boundary_edges)
    missing = sorted(set(tags) - set(boundary_conditions))
    if missing:
        raise ValueError(f"Boundary tags without a boundary condition: {missing}.")
    unknown = sorted(set(boundary_conditions) - set(tags))
    if unknown:
        raise ValueError(f"Boundary conditions for tags that are not in the mesh: {unknown}.")
    kinds = np.zeros(len(tags), dtype=np.int32)
    fixed_states = []
    for i, tag in enumerate(tags):
        bc = boundary_conditions[tag]
        if bc.kind not in (SLIP_WALL, FIXED_STATE):
            raise ValueError(f"Unsupported boundary condition for tag {tag!r}: {bc!r}.")
        kinds[i] = bc.kind
        if bc.kind == FIXED_STATE and len(mesh.boundary_edges[tag]):
            fixed_states.append(np.asarray(bc.state, dtype=np.float64))
    rows = np.unique(np.stack(fixed_states), axis=0) if fixed_states else np.zeros((0, 4))
    tag_row = np.zeros(len(tags), dtype=np.int32)
    for i, tag in enumerate(tags):
        bc = boundary_conditions[tag]
        if bc.kind == FIXED_STATE and len(rows):
            tag_row[i] = int(np.flatnonzero(np.all(rows == np.asarray(bc.state), axis=1))[0])
    return tags, kinds, tag_row, rows


class DeviceTables:
    """Mesh tables of one or more instances uploaded as torch tensors, plus the
    ``CfdMesh`` struct pointing at them. Keeps the tensors alive. Built from
    host tables (several instances), or on the GPU from one mesh
    (:meth:`build_on_device`)."""

    def __init__(self, parts: list[HostTables], device, precision: int):
        import torch

        self.device = torch.device(device)
        sizes = [p.num_elements for p in parts]
        # several instances: every instance starts at a multiple of LD_ALIGN
        # elements (padding elements carry instance -1), so that the tiled
        # kernels' blocks never straddle two instances
        spans = sizes if len(parts) == 1 else [padded_ld(n) for n in sizes]
        self.offsets = np.concatenate([[0], np.cumsum(spans)]).astype(np.int64)
        self.sizes = np.asarray(sizes, dtype=np.int64)
        k = int(self.offsets[-1]) if len(parts) == 1 else int(self.offsets[-2] + sizes[-1])
        ld = padded_ld(k)
        self.num_elements, self.ld, self.num_instances = k, ld, len(parts)
        bc_off = np.concatenate([[0], np.cumsum([len(p.bc_states) for p in parts])]).astype(np.int64)

        def cat(name, rows):
            out = np.zeros((rows, ld), dtype=getattr(parts[0], name).dtype)
            for p, o in zip(parts, self.offsets[:-1]):
                out[:, o:o + p.num_elements] = getattr(p, name).reshape(rows, -1)
            return out

        metric, face_geo, face_hlen = cat("metric", 4), cat("face_geo", 9), cat("face_hlen", 3)
        cs = cat("cs_coef", 6)
        dt_geo, jac = cat("dt_geo", 1)[0], cat("jacobian", 1)[0]
        nbr = np.zeros((3, ld), dtype=np.int32)
        info = np.zeros(ld, dtype=np.int32)
        inst = np.full(ld, -1, dtype=np.int32)
        for i, (p, o) in enumerate(zip(parts, self.offsets[:-1])):
            kinds = np.stack([(p.face_info >> (8 * f)) & 3 for f in range(3)])
            local = p.neighbor.astype(np.int64)
            glob = np.where(kinds >= FIXED_STATE, local + bc_off[i], np.where(kinds == 0, local + o, 0))
            nbr[:, o:o + p.num_elements] = glob
            info[o:o + p.num_elements] = p.face_info
            inst[o:o + p.num_elements] = i
        bcs = np.concatenate([p.bc_states for p in parts]) if bc_off[-1] else np.zeros((1, 4))

        t = lambda a: torch.as_tensor(np.ascontiguousarray(a)).to(self.device)  # noqa: E731
        self.metric, self.face_geo, self.face_hlen = t(metric), t(face_geo), t(face_hlen)
        self.dt_geo, self.jacobian, self.cs_coef = t(dt_geo), t(jac), t(cs)
        self.neighbor, self.face_info = t(nbr), t(info)
        self.instance = t(inst) if len(parts) > 1 else None
        self.bc_states = t(bcs)
        self._finish(precision)

    def _finish(self, precision: int) -> None:
        """FP32 copies (mixed form) and the CfdMesh struct."""
        self.precision = precision
        if precision == _native.CFD_FP32_MIXED:
            self.metric32 = self.metric.float().contiguous()
            self.face_geo32 = self.face_geo.float().contiguous()
            self.cs_coef32 = self.cs_coef.float().contiguous()
        else:
            self.metric32 = self.face_geo32 = self.cs_coef32 = None
        ptr = lambda x: None if x is None else x.data_ptr()  # noqa: E731
        self.struct = _native.CfdMesh(
            self.num_elements, self.ld, self.num_instances, 1 if self.num_instances > 1 else 0, ptr(self.metric),
            ptr(self.face_geo), ptr(self.face_hlen), ptr(self.dt_geo), ptr(self.jacobian), ptr(self.cs_coef),
            ptr(self.neighbor), ptr(self.face_info), ptr(self.instance), ptr(self.bc_states), ptr(self.metric32),
            ptr(self.face_geo32), ptr(self.cs_coef32))

    def with_precision(self, precision: int) -> "DeviceTables":
        """The same FP64 tables (shared, not copied) for another arithmetic form."""
        other = object.__new__(DeviceTables)
        for name in ("device", "offsets", "sizes", "num_elements", "ld", "num_instances", "metric", "face_geo",
                     "face_hlen", "dt_geo", "jacobian", "cs_coef", "neighbor", "face_info", "instance", "bc_states"):
            setattr(other, name, getattr(self, name))
        other._finish(precision)
        return other

    @classmethod
    def build_on_device(cls, mesh: TriangleMesh, boundary_conditions, reference, device, precision: int,
                        relative_tolerance: float = 1e-9) -> "DeviceTables":
        """One mesh's tables built by the GPU (cfd_mesh_build): geometry,
        connectivity and boundary tags, Cockburn-Shu coefficients and the
        face-node pairing check, bit for bit the host builder's tables. An
        invalid mesh is reported with the host builder's error. Exact-state
        boundaries (per-node rows evaluated by a Python function) take the
        host builder."""
        import ctypes as C

        import torch

        if any(getattr(bc, "kind", None) == EXACT_STATE for bc in boundary_conditions.values()):
            from .mesh import build_connectivity

            conn = build_connectivity(mesh)
            geo = element_geometry(mesh)
            kind, state = resolve_boundary_conditions(conn, boundary_conditions)
            part = host_tables(mesh, conn, geo, reference, kind, state, device=device,
                               boundary_conditions=boundary_conditions)
            return cls([part], device, precision)
        tags, kinds, tag_row, rows = boundary_tag_tables(mesh, boundary_conditions)
        dev = torch.device(device)
        k = mesh.num_elements
        ld = padded_ld(k)
        lib = _native.load()
        # copies: the mesh's arrays are read-only, which torch does not accept as tensor storage
        verts = torch.from_numpy(np.array(mesh.vertices, dtype=np.float64)).to(dev)
        elems = torch.from_numpy(np.array(mesh.elements, dtype=np.int64)).to(dev)
        edge_list = [np.asarray(mesh.boundary_edges[t], dtype=np.int64).reshape(-1, 2) for t in tags]
        edges = np.concatenate(edge_list) if edge_list else np.zeros((0, 2), np.int64)
        edge_tag = np.concatenate([np.full(len(e), i, np.int32) for i, e in enumerate(edge_list)]) if edge_list \
            else np.zeros(0, np.int32)
        t_edges = torch.as_tensor(np.ascontiguousarray(edges)).to(dev)
        t_tag = torch.as_tensor(edge_tag).to(dev)
        t_kind = torch.as_tensor(kinds).to(dev)
        t_row = torch.as_tensor(tag_row).to(dev)
        fn = np.asarray(reference.face_nodes)
        r, sv = reference.r[fn], reference.s[fn]
        bary = torch.as_tensor(np.ascontiguousarray(np.stack([-(r + sv) / 2, (1 + r) / 2, (1 + sv) / 2], axis=-1))).to(dev)

        self = object.__new__(cls)
        self.device = dev
        self.offsets = np.array([0, k], dtype=np.int64)
        self.sizes = np.array([k], dtype=np.int64)
        self.num_elements, self.ld, self.num_instances = k, ld, 1
        z = lambda *shape, dtype=torch.float64: torch.zeros(shape, dtype=dtype, device=dev)  # noqa: E731
        self.metric, self.face_geo, self.face_hlen = z(4, ld), z(9, ld), z(3, ld)
        self.dt_geo, self.jacobian, self.cs_coef = z(ld), z(ld), z(6, ld)
        self.neighbor, self.face_info = z(3, ld, dtype=torch.int32), z(ld, dtype=torch.int32)
        self.instance = None
        self.bc_states = torch.as_tensor(rows if len(rows) else np.zeros((1, 4))).to(dev)
        out = _native.CfdMesh(k, ld, 1, 0, self.metric.data_ptr(), self.face_geo.data_ptr(),
                              self.face_hlen.data_ptr(), self.dt_geo.data_ptr(), self.jacobian.data_ptr(),
                              self.cs_coef.data_ptr(), self.neighbor.data_ptr(), self.face_info.data_ptr(), None,
                              self.bc_states.data_ptr(), None, None, None)
        inp = _native.CfdMeshBuild(len(mesh.vertices), k, ld, len(edges), len(tags), 0, verts.data_ptr(),
                                   elems.data_ptr(), t_edges.data_ptr() if len(edges) else None,
                                   t_tag.data_ptr() if len(edges) else None, t_kind.data_ptr() if len(tags) else None,
                                   t_row.data_ptr() if len(tags) else None)
        nbytes = int(lib.cfd_mesh_build_work_bytes(k, len(edges)))
        work = torch.empty(nbytes, dtype=torch.uint8, device=dev)
        status = torch.zeros(1, dtype=torch.int32, device=dev)
        stream = torch.cuda.current_stream(dev).cuda_stream
        _native.check(lib.cfd_mesh_build(C.byref(inp), C.byref(out), bary.data_ptr(), float(relative_tolerance),
                                         work.data_ptr(), nbytes, status.data_ptr(), stream))
        code = int(status.item())
        if code:
            # the host builders raise the same errors with their messages
            from .mesh import build_connectivity

            conn = build_connectivity(mesh)
            geo = element_geometry(mesh)
            neighbor_coefficients(conn, geo)
            check_face_pairing(mesh, conn, reference, relative_tolerance, geometry=geo)
            raise ValueError(f"The mesh tables could not be built (status {code}).")
        self._finish(precision)
        return self
