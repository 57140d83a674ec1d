"""Case I/O around the step: gmsh meshes with named boundaries, VTK
snapshots, and initial states read from a file.

gmsh 2.2 ASCII (``read_gmsh`` / ``write_gmsh``).  The reference hands the
mesh file to PETSc (``DMPlexCreateFromFile``, ``VirtualSolver.hpp:386-389``),
which stores the physical tag of each boundary element in the "Face Sets"
label.  It then maps the tags to the model's boundary tags:

* ``MeshConfigLoader::loadBoundaryMapping`` (``MeshConfigLoader.hpp:15-42``)
  reads ``$PhysicalNames`` into name -> (dim, tag);
* every model tag except ``"default"`` must appear there with dimension
  ``dim - 1`` (``VirtualSolver.hpp:391-411``);
* model tag i takes the file's tag of its name, and ``"default"`` takes
  tag 1 when the file does not name it (``VirtualSolver.hpp:499-511``);
* a boundary face whose tag maps to no model tag gets no flux at all
  (``TransportStep.hpp:496-500``, ``Gradient.hpp:125``):
  ``FACE_NO_CONDITION`` here.

Snapshots (``write_vtu``, ``SnapshotWriter``).  The reference writes
``<filename>-NNN.vtu`` whenever t >= next_snap - 1e-9 dt_snap, with
dt_snap = t_end / snapshots (``IOManager.hpp:33-37, 60-79, 100-120``).  Each
file holds the cell state packed with the aux variables
(``VirtualSolver.hpp:359-384``).  It also keeps ``<filename>.vtu.series``
listing name and time (``IOManager.hpp:346-360``).  Here the cell data arrays
are "Q" (n_dof_q components) and "Aux" (n_dof_qaux), base64-encoded.

Initial states (``load_state``, ``overlay_state``).  The reference loads the
dataset "state" of an HDF5 file, whole or only the components listed in
``initial_condition_mask`` (``IOManager.hpp:122-192``), in the mesh's
natural cell order as its ``generate_ic.py`` writes it.  HDF5 files are read
by the library-free reader of ``hdf5.py`` (contiguous datasets, the layout
that script writes); ``.npy`` / ``.npz`` (key "state") hold the same array.
"""
from __future__ import annotations

import base64
import os
import xml.etree.ElementTree as ET
from typing import Dict, Optional, Sequence

import numpy as np

from . import mesh as meshmod
from .mesh import FACE_INTERIOR, FACE_NO_CONDITION, Mesh

# gmsh 2.2 element types -> (dimension, nodes)
_GMSH_TYPES = {15: (0, 1), 1: (1, 2), 2: (2, 3), 3: (2, 4)}


def _sections(path):
    with open(path) as f:
        lines = [ln.rstrip("\n") for ln in f]
    out, i = {}, 0
    while i < len(lines):
        s = lines[i].strip()
        if s.startswith("$") and not s.startswith("$End"):
            name = s[1:]
            j = i + 1
            while j < len(lines) and lines[j].strip() != "$End" + name:
                j += 1
            out[name] = lines[i + 1: j]
            i = j
        i += 1
    return out


def physical_names(path: str) -> Dict[str, tuple]:
    """name -> (dim, tag) from $PhysicalNames (MeshConfigLoader.hpp:15-42)."""
    sec = _sections(path).get("PhysicalNames")
    out = {}
    if not sec:
        return out
    for ln in sec[1:]:
        t = ln.split(None, 2)
        if len(t) < 3:
            continue
        try:
            dim, tag = int(t[0]), int(t[1])
        except ValueError:
            continue
        raw = t[2]
        a, b = raw.find('"'), raw.rfind('"')
        if a != -1 and b != -1:
            out[raw[a + 1: b]] = (dim, tag)
    return out


def boundary_map(names: Dict[str, tuple], boundary_tags: Sequence[str], dim: int) -> Dict[int, int]:
    """Physical tag -> model boundary index (VirtualSolver.hpp:391-411, 499-511);
    ValueError when a named model tag is missing or has the wrong dimension."""
    for n in boundary_tags:
        if n == "default":
            continue
        if n not in names or names[n][0] != dim - 1:
            raise ValueError("GMSH boundaries must exactly match model tags (excluding 'default'): "
                             "%r missing or not of dimension %d" % (n, dim - 1))
    out = {}
    for i, n in enumerate(boundary_tags):
        tag = names[n][1] if n in names else (1 if n == "default" else None)
        if tag is not None:
            out[tag] = i
    return out


def read_gmsh(path: str, boundary_tags: Sequence[str] = ("default",)) -> Mesh:
    """A gmsh 2.2 ASCII mesh: triangles and/or quadrilaterals (2-D; a mixed
    mesh becomes -1 padded [C, 4] cells) or segments (1-D) as cells, in file
    order; boundary faces carry the model boundary index of their element's
    physical tag, or FACE_NO_CONDITION."""
    sec = _sections(path)
    fmt = sec.get("MeshFormat", ["2.2 0 8"])[0].split()
    if not fmt[0].startswith("2") or (len(fmt) > 1 and fmt[1] != "0"):
        raise ValueError("%s: only gmsh 2.x ASCII files are read (MeshFormat %s)" % (path, " ".join(fmt)))
    nodes = sec["Nodes"]
    nv = int(nodes[0])
    ids = np.empty(nv, dtype=np.int64)
    xy = np.empty((nv, 2))
    for k, ln in enumerate(nodes[1: 1 + nv]):
        t = ln.split()
        ids[k] = int(t[0])
        xy[k] = float(t[1]), float(t[2])
    idmap = {int(v): k for k, v in enumerate(ids)}
    els = sec["Elements"]
    ne = int(els[0])
    by_dim = {0: [], 1: [], 2: []}
    for ln in els[1: 1 + ne]:
        t = [int(v) for v in ln.split()]
        et, nt = t[1], t[2]
        if et not in _GMSH_TYPES:
            raise ValueError("%s: gmsh element type %d is not supported" % (path, et))
        d, nn = _GMSH_TYPES[et]
        tag = t[3] if nt >= 1 else 0
        by_dim[d].append((et, tag, [idmap[v] for v in t[3 + nt: 3 + nt + nn]]))
    dim = 2 if by_dim[2] else 1
    cells = by_dim[dim]
    if dim == 2:
        types = {e[0] for e in cells}
        if types == {2}:
            conn = np.array([e[2] for e in cells], dtype=np.int64)
            m = meshmod.from_triangles(xy, conn, name=path, boundary_bc=FACE_NO_CONDITION)
        else:   # quadrilaterals, or a mix with triangles padded by -1
            conn = np.array([e[2] + [-1] * (4 - len(e[2])) for e in cells], dtype=np.int64)
            m = meshmod.from_polygons(xy, conn, name=path, boundary_bc=FACE_NO_CONDITION)
    else:
        seg = np.array([e[2] for e in cells], dtype=np.int64)
        chain = np.all(seg[1:, 0] == seg[:-1, 1]) and np.all(np.diff(xy[np.append(seg[:, 0], seg[-1, 1]), 0]) > 0)
        if not chain:
            raise ValueError("%s: 1-D segments must follow each other in increasing x" % path)
        m = meshmod.interval(xy[np.append(seg[:, 0], seg[-1, 1]), 0], name=path,
                             bc_left=FACE_NO_CONDITION, bc_right=FACE_NO_CONDITION)
    bmap = boundary_map(physical_names(path), list(boundary_tags), dim)
    fv = meshmod.face_vertices(m)
    if dim == 2:
        key = {(min(e[2]), max(e[2])): e[1] for e in by_dim[1]}
        fkeys = [(int(a), int(b)) for a, b in fv]
    else:
        # interval() keeps the chain's nodes in order: vertex k of the mesh is chain node k
        pos = {int(v): k for k, v in enumerate(np.append(seg[:, 0], seg[-1, 1]))}
        key = {pos[e[2][0]]: e[1] for e in by_dim[0] if e[2][0] in pos}
        fkeys = [int(v) for v in fv]
    bc = m.face_bc.copy()
    for f in np.nonzero(m.face_cells[:, 1] < 0)[0]:
        tag = key.get(fkeys[f])
        bc[f] = bmap.get(tag, FACE_NO_CONDITION) if tag is not None else FACE_NO_CONDITION
    m.face_bc = bc.astype(np.int32)
    return m


def write_gmsh(path: str, mesh: Mesh, face_tags: Optional[np.ndarray] = None,
               names: Optional[Dict[int, str]] = None):
    """gmsh 2.2 ASCII: the boundary faces with face_tags[f] > 0 as elements of
    that physical tag (default: every boundary face, tag 1), names: tag ->
    physical name of the boundary tags (default {1: "boundary"}), then the
    cells under one more "domain" tag."""
    F = mesh.n_faces
    bnd = mesh.face_cells[:, 1] < 0
    if face_tags is None:
        face_tags = np.where(bnd, 1, 0)
    face_tags = np.asarray(face_tags, dtype=np.int64)
    names = dict(names) if names is not None else {1: "boundary"}
    dom_tag = max([0] + list(names) + [int(face_tags.max()) if F else 0]) + 1
    fv = meshmod.face_vertices(mesh)
    bfaces = [f for f in range(F) if bnd[f] and face_tags[f] > 0]
    V = mesh.vertices.shape[0]
    nvc = (mesh.cells >= 0).sum(1)
    if mesh.dim == 2:
        ctypes = [{3: 2, 4: 3}[int(n)] for n in nvc]      # triangle, quadrilateral
        btype = 1
    else:
        ctypes, btype = [1] * mesh.n_cells, 15
    with open(path, "w") as f:
        f.write("$MeshFormat\n2.2 0 8\n$EndMeshFormat\n")
        f.write("$PhysicalNames\n%d\n" % (len(names) + 1))
        for tag in sorted(names):
            f.write('%d %d "%s"\n' % (mesh.dim - 1, tag, names[tag]))
        f.write('%d %d "domain"\n$EndPhysicalNames\n' % (mesh.dim, dom_tag))
        f.write("$Nodes\n%d\n" % V)
        for i, (x, y) in enumerate(mesh.vertices):
            f.write("%d %.17g %.17g 0.0\n" % (i + 1, x, y))
        f.write("$EndNodes\n$Elements\n%d\n" % (len(bfaces) + mesh.n_cells))
        k = 1
        for fc in bfaces:
            vs = fv[fc] if mesh.dim == 2 else [fv[fc]]
            f.write("%d %d 2 %d %d %s\n" % (k, btype, face_tags[fc], face_tags[fc],
                                            " ".join(str(int(v) + 1) for v in vs)))
            k += 1
        for c, ct in zip(mesh.cells, ctypes):
            f.write("%d %d 2 %d %d %s\n" % (k, ct, dom_tag, dom_tag, " ".join(str(int(v) + 1) for v in c if v >= 0)))
            k += 1
        f.write("$EndElements\n")


# ------------------------------------------------------------------ VTK
_VTK_TYPE = {(1, 2): 3, (2, 3): 5, (2, 4): 9}     # line, triangle, quad


def _b64(a: np.ndarray) -> str:
    raw = np.ascontiguousarray(a).tobytes()
    return base64.b64encode(np.uint64(len(raw)).tobytes() + raw).decode("ascii")


def write_vtu(path: str, mesh: Mesh, q: np.ndarray, aux: Optional[np.ndarray] = None, time: float = 0.0):
    """VTK XML unstructured grid: the mesh with cell data "Q" (and "Aux"),
    binary base64 with 64-bit headers, and the time as field data."""
    C, K = mesh.cells.shape
    pts = np.zeros((mesh.vertices.shape[0], 3))
    pts[:, :2] = mesh.vertices
    q = np.asarray(q, dtype=np.float64).reshape(C, -1)

    def arr(parent, name, data, ncomp=None, vtype="Float64"):
        a = ET.SubElement(parent, "DataArray", type=vtype, Name=name, format="binary")
        if ncomp:
            a.set("NumberOfComponents", str(ncomp))
        a.text = _b64(data)

    root = ET.Element("VTKFile", type="UnstructuredGrid", version="1.0", byte_order="LittleEndian",
                      header_type="UInt64")
    grid = ET.SubElement(root, "UnstructuredGrid")
    fd = ET.SubElement(grid, "FieldData")
    t = ET.SubElement(fd, "DataArray", type="Float64", Name="TIME", NumberOfTuples="1", format="ascii")
    t.text = repr(float(time))
    piece = ET.SubElement(grid, "Piece", NumberOfPoints=str(pts.shape[0]), NumberOfCells=str(C))
    pe = ET.SubElement(piece, "Points")
    arr(pe, "Points", pts, 3)
    ce = ET.SubElement(piece, "Cells")
    nvc = (mesh.cells >= 0).sum(1)                      # -1 padded rows: mixed cells
    arr(ce, "connectivity", mesh.cells[mesh.cells >= 0].astype(np.int64), vtype="Int64")
    arr(ce, "offsets", np.cumsum(nvc).astype(np.int64), vtype="Int64")
    arr(ce, "types", np.array([_VTK_TYPE[(mesh.dim, int(n))] for n in nvc], dtype=np.uint8), vtype="UInt8")
    cd = ET.SubElement(piece, "CellData", Scalars="Q")
    arr(cd, "Q", q, q.shape[1])
    if aux is not None:
        a = np.asarray(aux, dtype=np.float64).reshape(C, -1)
        arr(cd, "Aux", a, a.shape[1])
    ET.ElementTree(root).write(path, xml_declaration=True, encoding="utf-8")


def read_vtu_cell_data(path: str) -> Dict[str, np.ndarray]:
    """The binary arrays of a file written by write_vtu by name; arrays with a
    component count come back as [n, ncomp] (cell data "Q", "Aux", points)."""
    root = ET.parse(path).getroot()
    out = {}
    for a in root.iter("DataArray"):
        if a.get("format") != "binary":
            continue
        raw = base64.b64decode(a.text)
        n = int(np.frombuffer(raw[:8], dtype=np.uint64)[0])
        dt = {"Float64": np.float64, "Int64": np.int64, "UInt8": np.uint8}[a.get("type")]
        v = np.frombuffer(raw[8: 8 + n], dtype=dt)
        nc = a.get("NumberOfComponents")
        out[a.get("Name")] = v.reshape(-1, int(nc)) if nc is not None else v
    return out


class SnapshotWriter:
    """Snapshots at t = 0, dt_snap, 2 dt_snap, ... (dt_snap = t_end /
    snapshots) as <directory>/<filename>-NNN.vtu plus the .vtu.series index
    (IOManager.hpp:33-79, 100-120, 346-360).  The reference's "snap",
    "interpolate" and default logics all advance next_snap by dt_snap; its
    "loose" logic loops without end (`while (next <= next + dt)`) and is not
    offered."""

    def __init__(self, directory: str, filename: str, t_end: float, snapshots: int = 10,
                 clean_directory: bool = False):
        if snapshots < 1:
            raise ValueError("snapshots must be >= 1")
        self.directory, self.filename = directory, filename
        self.dt_snap = t_end / snapshots
        self.next_snap = 0.0
        self.index = 0
        self.log = []
        os.makedirs(directory, exist_ok=True)
        if clean_directory:
            for e in os.listdir(directory):
                p = os.path.join(directory, e)
                if os.path.isfile(p):
                    os.remove(p)

    def should_write(self, time: float, force: bool = False) -> bool:
        return force or time >= self.next_snap - 1e-9 * self.dt_snap

    def write(self, mesh: Mesh, q: np.ndarray, aux: Optional[np.ndarray], time: float):
        name = "%s-%03d.vtu" % (self.filename, self.index)
        write_vtu(os.path.join(self.directory, name), mesh, q, aux, time)
        self.log.append((name, float(time)))
        with open(os.path.join(self.directory, self.filename + ".vtu.series"), "w") as f:
            f.write('{\n  "file-series-version" : "1.0",\n  "files" : [\n')
            for i, (n, t) in enumerate(self.log):
                f.write('    { "name" : "%s", "time" : %.6e }%s\n' % (n, t, "," if i < len(self.log) - 1 else ""))
            f.write("  ]\n}\n")

    def advance(self):
        self.next_snap += self.dt_snap
        self.index += 1

    def monitor(self, solver, mesh: Mesh, time: float):
        """VirtualSolver::Monitor (VirtualSolver.hpp:181-186): write and advance when due."""
        if self.should_write(time):
            self.write(mesh, solver.get_state(), solver.get_aux(), time)
            self.advance()


def run_with_snapshots(solver, mesh: Mesh, writer: SnapshotWriter, t_end: float, max_steps: int = 1 << 30) -> int:
    """The reference's step loop with its monitor (MUSCLSolver.hpp:120-186):
    a snapshot check at the start and after every step, until t_end.
    Returns the steps taken."""
    t, _ = solver.time()
    writer.monitor(solver, mesh, t)
    n = 0
    while t < t_end and n < max_steps:
        solver.step(1)
        n += 1
        t, _ = solver.time()
        writer.monitor(solver, mesh, t)
    return n


# ------------------------------------------------------------ initial states
def load_state(path: str, n_cells: Optional[int] = None, n_dof_q: Optional[int] = None) -> np.ndarray:
    """The "state" array of an initial-condition file (natural cell order):
    HDF5 (.h5 / .hdf5: dataset "state", flat cell-major float64 with the
    num_components attribute, as the reference's generate_ic.py writes it;
    returned as [C, n_components]), .npy, or .npz with key "state" ([C,
    n_dof_q] or flat).  n_cells / n_dof_q check or supply the shape."""
    if path.endswith((".h5", ".hdf5")):
        from . import hdf5

        return hdf5.read_state(path, n_cells=n_cells, n_dof_q=n_dof_q)
    if path.endswith(".npy"):
        return np.load(path)
    if path.endswith(".npz"):
        with np.load(path) as z:
            return z["state"]
    raise ValueError("%s: initial states are read from .h5 / .hdf5 ('state'), .npy or .npz ('state')" % path)


def overlay_state(q: np.ndarray, loaded: np.ndarray, mask: Sequence[int] = ()) -> np.ndarray:
    """IOManager::LoadSolution (IOManager.hpp:145-183): the whole loaded state,
    or with a mask only those components over q."""
    q = np.array(q, dtype=np.float64)
    loaded = np.asarray(loaded, dtype=np.float64).reshape(q.shape)
    if not len(mask):
        return loaded.copy()
    for comp in mask:
        if 0 <= comp < q.shape[1]:
            q[:, comp] = loaded[:, comp]
    return q


def boundary_counts(mesh: Mesh) -> Dict[int, int]:
    """Boundary faces per bc index (FACE_NO_CONDITION included)."""
    b = mesh.face_bc[mesh.face_cells[:, 1] < 0]
    return {int(k): int((b == k).sum()) for k in np.unique(b)}


__all__ = ["read_gmsh", "write_gmsh", "physical_names", "boundary_map", "write_vtu", "read_vtu_cell_data",
           "SnapshotWriter", "run_with_snapshots", "load_state", "overlay_state", "boundary_counts",
           "FACE_INTERIOR", "FACE_NO_CONDITION"]
