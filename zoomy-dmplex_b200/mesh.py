"""Unstructured meshes and their finite-volume geometry.

The reference reads a gmsh file into a PETSc DMPlex and takes its cell-centred
finite-volume geometry from ``DMPlexGetGeometryFVM`` (reference
``VirtualSolver.hpp:386-525``, ``TransportStep.hpp:388-410``).  This module
builds the same quantities without PETSc:

* faces are numbered in first-encounter order over the cells, each cell's faces
  in its local edge order ``(v0,v1), (v1,v2), (v2,v0)`` -- the order DMPlex
  interpolation produces -- so ``face_cells[f, 0]`` (the support's first cell)
  is the lower-numbered cell;
* face normals are area-weighted (length = face measure) and oriented from
  ``face_cells[f, 0]`` to ``face_cells[f, 1]``; on the boundary they point out;
* ``cell_faces`` is the cell's cone (local edge order) and ``cell_nbrs`` its
  face-neighbour list in cone order, i.e. what ``DMPlexGetAdjacency`` returns
  for a finite-volume field (cells sharing a face, reference
  ``TransportStep.hpp:106-120``);
* boundary faces carry a boundary-condition index (``face_bc``): the
  reference maps every exterior face of an untagged mesh to the model's
  ``"default"`` tag, index 0 (``VirtualSolver.hpp:499-511``).

Meshes of the benchmark configurations are seeded jittered-grid Delaunay
triangulations of the unit square (``jittered_square``); 1-D interval meshes
(``interval``) and gmsh 2.2 files (``read_msh``/``write_msh``) are supported
as well.
"""
from __future__ import annotations

import dataclasses
from typing import Optional

import numpy as np

FACE_INTERIOR = -1
FACE_NO_CONDITION = -2


@dataclasses.dataclass
class Mesh:
    dim: int                      # 1 or 2
    vertices: np.ndarray          # [V, 2]
    cells: np.ndarray             # [C, K] vertex ids (K = 2 segments, 3 triangles, 4 quadrilaterals; -1 padded)
    cell_centroid: np.ndarray     # [C, 2]
    cell_volume: np.ndarray       # [C]
    cell_faces: np.ndarray        # [C, K] int32, cone order
    face_cells: np.ndarray        # [F, 2] int32, [:,1] = -1 on the boundary
    face_centroid: np.ndarray     # [F, 2]
    face_normal: np.ndarray       # [F, 2] area-weighted, oriented cells[0] -> cells[1]
    face_bc: np.ndarray           # [F] int32: -1 interior, >= 0 bc index, -2 none
    name: str = "mesh"
    cell_cfl_skip: Optional[np.ndarray] = None   # [C] nonzero: left out of the CFL minimum (halo cells)

    @property
    def n_cells(self):
        return int(self.cells.shape[0])

    @property
    def n_faces(self):
        return int(self.face_cells.shape[0])

    @property
    def max_faces(self):
        return int(self.cell_faces.shape[1])

    def cell_nbrs(self):
        """Face neighbours of each cell in cone order, -1 padded ([C, K])."""
        f = self.cell_faces
        fc = self.face_cells[f]                       # [C, K, 2]
        me = np.arange(self.n_cells)[:, None]
        other = np.where(fc[..., 0] == me, fc[..., 1], fc[..., 0])
        other = np.where(f < 0, -1, other)
        # compact: boundary slots move to the end, cone order kept
        out = np.full_like(other, -1)
        cnt = np.zeros(self.n_cells, dtype=np.int64)
        for k in range(other.shape[1]):
            v = other[:, k]
            ok = v >= 0
            out[np.nonzero(ok)[0], cnt[ok]] = v[ok]
            cnt += ok
        return out.astype(np.int32)

    def inradius_proxy(self):
        """r_c = min over the cell's faces of |x_c - x_f| (reference
        ``VirtualSolver.hpp:329-340``)."""
        f = self.cell_faces
        d = self.face_centroid[np.maximum(f, 0)] - self.cell_centroid[:, None, :]
        r = np.sqrt((d[..., : self.dim] ** 2).sum(-1))
        r = np.where(f < 0, np.inf, r)
        return r.min(axis=1)

    def as_abi_arrays(self):
        """Contiguous arrays in the layout the C ABI (``zsme_mesh``) takes."""
        return dict(
            dim=self.dim,
            n_cells=self.n_cells,
            n_faces=self.n_faces,
            max_faces=self.max_faces,
            cell_centroid=np.ascontiguousarray(self.cell_centroid, dtype=np.float64),
            cell_volume=np.ascontiguousarray(self.cell_volume, dtype=np.float64),
            cell_faces=np.ascontiguousarray(self.cell_faces, dtype=np.int32),
            face_cells=np.ascontiguousarray(self.face_cells, dtype=np.int32),
            face_centroid=np.ascontiguousarray(self.face_centroid, dtype=np.float64),
            face_normal=np.ascontiguousarray(self.face_normal, dtype=np.float64),
            face_bc=np.ascontiguousarray(self.face_bc, dtype=np.int32),
            **({} if self.cell_cfl_skip is None
               else {"cell_cfl_skip": np.ascontiguousarray(self.cell_cfl_skip, dtype=np.uint8)}),
        )


# ---------------------------------------------------------------------------
# construction
# ---------------------------------------------------------------------------
def _vertex_counts(cells: np.ndarray) -> np.ndarray:
    """Vertices of each polygon in a -1 padded [C, K] array (padding only at
    the end of a row)."""
    ok = cells >= 0
    nv = ok.sum(1)
    if not np.array_equal(ok, np.arange(cells.shape[1])[None, :] < nv[:, None]):
        raise ValueError("polygon rows must list their vertices first and pad with -1")
    return nv


def _faces_from_cells(cells: np.ndarray, nloc: int):
    """First-encounter face numbering (cell order, then local face order).
    2-D: local face k of a cell is its edge (v_k, v_(k+1) mod n) over its n
    vertices (rows of -1 padded polygons have fewer faces; their missing
    slots get face -1).  Returns the [C, nloc] face ids, the [F, 2] support
    and, per face, the flat index c * nloc + k of its first encounter."""
    C = cells.shape[0]
    if nloc >= 3:  # polygon edges (v_k, v_k+1)
        nv = _vertex_counts(cells)
        k = np.arange(nloc)[None, :]
        valid = k < nv[:, None]
        a = np.where(valid, cells, 0)
        b = np.take_along_axis(a, (k + 1) % nv[:, None], axis=1)
        pos = np.nonzero(valid.reshape(-1))[0]
        lo = np.minimum(a, b).reshape(-1)[pos].astype(np.int64)
        hi = np.maximum(a, b).reshape(-1)[pos].astype(np.int64)
        key = lo * (int(cells.max()) + 1) + hi
    else:  # 1-D: faces are the vertices
        pos = np.arange(C * nloc)
        key = cells.reshape(-1).astype(np.int64)
    uniq, first, inv = np.unique(key, return_index=True, return_inverse=True)
    order = np.argsort(first, kind="stable")           # face ids by first encounter
    rank = np.empty_like(order)
    rank[order] = np.arange(order.size)
    fid = np.full(C * nloc, -1, dtype=np.int64)
    fid[pos] = rank[inv]
    F = uniq.size
    flat_c = pos // nloc
    flat_f = fid[pos]
    # support: the encountering cells in cell order
    srt = np.lexsort((flat_c, flat_f))
    ff, cc = flat_f[srt], flat_c[srt]
    face_cells = np.full((F, 2), -1, dtype=np.int64)
    start = np.searchsorted(ff, np.arange(F))
    face_cells[:, 0] = cc[start]
    cnt = np.bincount(ff, minlength=F)
    if (cnt > 2).any():
        raise ValueError("non-manifold mesh: a face has more than two cells")
    two = cnt == 2
    face_cells[two, 1] = cc[start[two] + 1]
    return fid.reshape(C, nloc).astype(np.int32), face_cells.astype(np.int32), pos[first[order]]


def from_triangles(vertices: np.ndarray, tris: np.ndarray, name="mesh", boundary_bc=0) -> Mesh:
    vertices = np.asarray(vertices, dtype=np.float64)[:, :2].copy()
    tris = np.asarray(tris, dtype=np.int64).copy()
    p0, p1, p2 = vertices[tris[:, 0]], vertices[tris[:, 1]], vertices[tris[:, 2]]
    area2 = (p1[:, 0] - p0[:, 0]) * (p2[:, 1] - p0[:, 1]) - (p1[:, 1] - p0[:, 1]) * (p2[:, 0] - p0[:, 0])
    keep = np.abs(area2) > 1e-14 * np.abs(area2).max()
    tris = tris[keep]
    area2 = area2[keep]
    neg = area2 < 0                                     # orient counter-clockwise
    tris[neg] = tris[neg][:, [0, 2, 1]]
    p0, p1, p2 = vertices[tris[:, 0]], vertices[tris[:, 1]], vertices[tris[:, 2]]
    centroid = (p0 + p1 + p2) / 3.0
    volume = 0.5 * np.abs(area2)
    cell_faces, face_cells, first = _faces_from_cells(tris, 3)
    C = tris.shape[0]
    loc = first % 3                                     # local edge of the first cell
    c0 = face_cells[:, 0]
    va = tris[c0, loc]
    vb = tris[c0, (loc + 1) % 3]
    xa, xb = vertices[va], vertices[vb]
    fcent = 0.5 * (xa + xb)
    e = xb - xa
    normal = np.stack([e[:, 1], -e[:, 0]], axis=1)
    out = ((fcent - centroid[c0]) * normal).sum(1) < 0
    normal[out] *= -1.0
    bc = np.where(face_cells[:, 1] < 0, boundary_bc, FACE_INTERIOR).astype(np.int32)
    return Mesh(2, vertices, tris.astype(np.int32), centroid, volume, cell_faces, face_cells,
                fcent, normal, bc, name=name)


def from_polygons(vertices: np.ndarray, polys: np.ndarray, name="mesh", boundary_bc=0) -> Mesh:
    """Mesh of convex polygons, [C, K] vertex ids, rows with fewer than K
    vertices padded with -1 at the end (mixed triangles and quadrilaterals;
    such a cell has -1 face slots).  Counter-clockwise or clockwise
    (re-oriented counter-clockwise): shoelace areas and centroids, edge
    midpoints and outward edge normals."""
    vertices = np.asarray(vertices, dtype=np.float64)[:, :2].copy()
    polys = np.asarray(polys, dtype=np.int64).copy()
    K = polys.shape[1]
    nv = _vertex_counts(polys)
    if (nv < 3).any():
        raise ValueError("a polygon needs at least 3 vertices")
    k = np.arange(K)[None, :]
    valid = k < nv[:, None]
    nxt = (k + 1) % nv[:, None]

    def shoelace(pl):
        P = vertices[np.where(valid, pl, 0)]              # [C, K, 2]
        Pn = np.take_along_axis(P, np.broadcast_to(nxt[..., None], P.shape), axis=1)
        cross = np.where(valid, P[:, :, 0] * Pn[:, :, 1] - Pn[:, :, 0] * P[:, :, 1], 0.0)
        return P, Pn, cross

    _, _, cross = shoelace(polys)
    neg = cross.sum(1) < 0
    rev = np.where(valid, nv[:, None] - 1 - k, k)         # reverse the listed vertices
    polys[neg] = np.take_along_axis(polys[neg], rev[neg], axis=1)
    P, Pn, cross = shoelace(polys)
    area2 = cross.sum(1)
    centroid = ((P + Pn) * cross[:, :, None]).sum(1) / (3.0 * area2[:, None])
    volume = 0.5 * area2
    cell_faces, face_cells, first = _faces_from_cells(polys, K)
    loc = first % K
    c0 = face_cells[:, 0]
    xa = vertices[polys[c0, loc]]
    xb = vertices[polys[c0, (loc + 1) % nv[c0]]]
    fcent = 0.5 * (xa + xb)
    e = xb - xa
    normal = np.stack([e[:, 1], -e[:, 0]], axis=1)
    out = ((fcent - centroid[c0]) * normal).sum(1) < 0
    normal[out] *= -1.0
    bc = np.where(face_cells[:, 1] < 0, boundary_bc, FACE_INTERIOR).astype(np.int32)
    return Mesh(2, vertices, polys.astype(np.int32), centroid, volume, cell_faces, face_cells,
                fcent, normal, bc, name=name)


def pad_face_slots(mesh: Mesh, K: int) -> Mesh:
    """The same mesh with K face slots per cell: cells and cell_faces padded
    with -1 columns (a triangle mesh taken to K = 4 joins quadrilateral or
    mixed meshes in one ensemble).  The geometry, face numbering and each
    cell's faces are unchanged, so the step is unchanged too."""
    k0 = mesh.max_faces
    if K == k0:
        return mesh
    if K < k0 or mesh.dim != 2:
        raise ValueError("can only add face slots to a 2-D mesh (%d -> %d)" % (k0, K))
    pad = np.full((mesh.n_cells, K - k0), -1, dtype=np.int32)
    return dataclasses.replace(mesh, cells=np.concatenate([mesh.cells.astype(np.int32), pad], 1),
                               cell_faces=np.concatenate([mesh.cell_faces.astype(np.int32), pad], 1))


def mixed_square(n: int, seed: int = 0, jitter: float = 0.2, name=None) -> Mesh:
    """Mixed triangles and quadrilaterals on the unit square: an n x n grid
    with interior nodes jittered by +-jitter * spacing (seeded), every other
    quadrilateral (checkerboard) split into two triangles along alternating
    diagonals; -1 padded [C, 4] cells, so triangle cells have one empty face
    slot."""
    rng = np.random.default_rng(seed)
    x = np.linspace(0.0, 1.0, n + 1)
    X, Y = np.meshgrid(x, x, indexing="ij")
    h = 1.0 / n
    inner = np.zeros_like(X, dtype=bool)
    inner[1:-1, 1:-1] = True
    X = X + np.where(inner, rng.uniform(-jitter, jitter, X.shape) * h, 0.0)
    Y = Y + np.where(inner, rng.uniform(-jitter, jitter, Y.shape) * h, 0.0)
    verts = np.stack([X.reshape(-1), Y.reshape(-1)], 1)
    idx = lambda i, j: i * (n + 1) + j
    polys = []
    for i in range(n):
        for j in range(n):
            a, b, c, d = idx(i, j), idx(i + 1, j), idx(i + 1, j + 1), idx(i, j + 1)
            if (i + j) % 2 == 0:
                polys.append([a, b, c, d])
            elif (i // 2 + j) % 2 == 0:
                polys += [[a, b, c, -1], [a, c, d, -1]]
            else:
                polys += [[a, b, d, -1], [b, c, d, -1]]
    return from_polygons(verts, np.array(polys), name=name or "mixed%d" % n)


def quad_strip(x: np.ndarray, height: float = 1.0, name="strip") -> Mesh:
    """One row of rectangles [x_i, x_i+1] x [0, height] (walls all round):
    with height 1 and a state uniform in y with v = 0, the 2-D scheme reduces
    to the 1-D scheme on the interval mesh of the same nodes."""
    x = np.asarray(x, dtype=np.float64)
    n = x.size - 1
    verts = np.concatenate([np.stack([x, np.zeros_like(x)], 1), np.stack([x, np.full_like(x, height)], 1)])
    i = np.arange(n)
    quads = np.stack([i, i + 1, n + 2 + i, n + 1 + i], axis=1)
    m = from_polygons(verts, quads, name=name)
    # rectangle measures formed exactly as interval() forms the 1-D ones
    m.cell_volume = np.abs(x[1:] - x[:-1]) * height
    m.cell_centroid = np.stack([0.5 * (x[:-1] + x[1:]), np.full(n, 0.5 * height)], axis=1)
    return m


def jittered_square(n: int, seed: int = 0, jitter: float = 0.2, name=None) -> Mesh:
    """Delaunay triangulation of an n x n point grid on the unit square whose
    interior points are jittered uniformly by +-jitter*spacing (seeded); the
    boundary points stay on the boundary so the walls are straight."""
    from scipy.spatial import Delaunay

    rng = np.random.default_rng(seed)
    s = np.linspace(0.0, 1.0, n)
    X, Y = np.meshgrid(s, s, indexing="xy")
    pts = np.stack([X.ravel(), Y.ravel()], axis=1)
    h = 1.0 / (n - 1)
    interior = (pts[:, 0] > 0) & (pts[:, 0] < 1) & (pts[:, 1] > 0) & (pts[:, 1] < 1)
    jit = rng.uniform(-jitter * h, jitter * h, size=pts.shape)
    pts = pts + jit * interior[:, None]
    tri = Delaunay(pts)
    return from_triangles(pts, tri.simplices, name=name or "square_%d_s%d" % (n, seed))


def interval(x: np.ndarray, name="interval", bc_left=0, bc_right=0) -> Mesh:
    """1-D mesh of segments between sorted node coordinates x."""
    x = np.asarray(x, dtype=np.float64)
    V = x.size
    verts = np.stack([x, np.zeros(V)], axis=1)
    segs = np.stack([np.arange(V - 1), np.arange(1, V)], axis=1)
    cell_faces, face_cells, first = _faces_from_cells(segs, 2)
    centroid = 0.5 * (verts[segs[:, 0]] + verts[segs[:, 1]])
    volume = np.abs(x[1:] - x[:-1])
    vid = segs.reshape(-1)[first]
    fcent = verts[vid]
    normal = np.zeros((face_cells.shape[0], 2))
    c0 = face_cells[:, 0]
    normal[:, 0] = np.where(fcent[:, 0] >= centroid[c0, 0], 1.0, -1.0)
    bc = np.full(face_cells.shape[0], FACE_INTERIOR, dtype=np.int32)
    bnd = face_cells[:, 1] < 0
    bc[bnd & (fcent[:, 0] <= x.min())] = bc_left
    bc[bnd & (fcent[:, 0] >= x.max())] = bc_right
    return Mesh(1, verts, segs.astype(np.int32), centroid, volume, cell_faces, face_cells,
                fcent, normal, bc, name=name)


def face_vertices(mesh: Mesh) -> np.ndarray:
    """Vertex ids of each face: [F, 2] (lower id first) in 2-D, [F] in 1-D.
    A cell's local face k is its edge (v_k, v_(k+1) mod n) over its n
    vertices (-1 padded rows), or its vertex v_k in 1-D."""
    C, K = mesh.cell_faces.shape
    f = mesh.cell_faces.reshape(-1)
    c = np.repeat(np.arange(C), K)
    k = np.tile(np.arange(K), C)
    ok = f >= 0
    f, c, k = f[ok], c[ok], k[ok]
    a = mesh.cells[c, k].astype(np.int64)
    if mesh.dim == 1:
        out = np.empty(mesh.n_faces, dtype=np.int64)
        out[f] = a
        return out
    nv = (mesh.cells >= 0).sum(1)
    b = mesh.cells[c, (k + 1) % nv[c]].astype(np.int64)
    out = np.empty((mesh.n_faces, 2), dtype=np.int64)
    out[f, 0] = np.minimum(a, b)
    out[f, 1] = np.maximum(a, b)
    return out


# ---------------------------------------------------------------------------
# gmsh 2.2 ASCII (the format of the reference's meshes): see caseio
# ---------------------------------------------------------------------------
def write_msh(path: str, mesh: Mesh, **kw):
    from .caseio import write_gmsh

    write_gmsh(path, mesh, **kw)


def read_msh(path: str, boundary_tags=("default",)) -> Mesh:
    from .caseio import read_gmsh

    return read_gmsh(path, boundary_tags)
