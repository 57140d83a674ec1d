"""Spatial partition of one mesh over several solvers with halo exchange.

The reference distributes its mesh with PETSc (DMPlexDistribute with
overlap, ``VirtualSolver.hpp:221``) and refreshes ghost cells with
global-to-local scatters in every right-hand-side evaluation
(``TransportStep.hpp:325-333``).  Here each part is a mesh of its own, run
by an unmodified solver handle:

* the part owns a set of cells (recursive coordinate bisection of the cell
  centroids, balanced by cell count) and carries a halo of every cell within
  ``halo_layers`` face-neighbour layers of them;
* one SSP-RK(s,2) stage updates a cell from the face states of its faces,
  which need the gradient and limiter bounds of its neighbours, so a stage
  reads two cell layers and an order-2 step 2 s layers (one layer per stage
  at order 1).  With that many halo layers every owned cell of a part ends a
  step with exactly the value of the undivided run; the outer halo layers
  hold stale values, which the exchange after the step overwrites;
* faces keep their global order and orientation, so every cell sums its
  faces in the same order as in the whole mesh; a face cut off at the
  halo's outer edge carries no flux (``FACE_NO_CONDITION``), oriented out of
  its one remaining cell;
* halo cells are left out of the CFL minimum (``cell_cfl_skip``), and the
  step's dt is the minimum over the parts of their CFL dts -- the dt of the
  whole mesh, because rounding cfl * ratio is monotone;
* after each step every part sends the owned cells that lie in another
  part's halo (``zsme_get_cells`` / ``zsme_set_cells``).

``PartitionedSolver`` runs all parts in one process (one GPU, host-side
exchange); ``exchange`` is the same schedule over ``torch.distributed``
point-to-point messages for one part per rank.

``PartRunner`` is the device-resident form: a part's step loop -- the
global dt as an all-reduce with MIN of the parts' CFL dts (the reference's
``MPI_Allreduce``, ``VirtualSolver.hpp:349``), the step at that dt, the halo
refresh -- as tensor operations in stream order.  With ``DevicePart`` (a
solver handle; halo cells packed and unpacked on the GPU by
``zsme_get_cells`` / ``zsme_set_cells`` on device buffers, the dt read and
imposed through ``zsme_get_time_device`` / ``zsme_step_dt_device``) and
``TorchComm`` over NCCL, nothing in a step synchronises the host: the
collectives are issued on the handle's stream, NCCL sends each packed halo
straight into the receiver's own receive buffer, and the receiver unpacks
it into its ghost cells.  ``LocalComm`` performs the same schedule for
several parts held by one process.
"""
from __future__ import annotations

import dataclasses
from typing import Dict, List, Optional

import numpy as np

from .mesh import FACE_INTERIOR, FACE_NO_CONDITION, Mesh


def halo_layers(reconstruction_order: int, ssp_stages: int) -> int:
    """Cell layers one step reads beyond a cell: 2 per stage at order 2
    (face states need the neighbours' gradients and bounds), 1 per stage at
    order 1 (forward Euler, one stage)."""
    return 2 * ssp_stages if reconstruction_order >= 2 else 1


def partition_cells(mesh: Mesh, nparts: int) -> np.ndarray:
    """Part of each cell: recursive coordinate bisection of the centroids
    (split along the longer extent, sizes proportional to the part counts)."""
    part = np.zeros(mesh.n_cells, dtype=np.int64)

    def split(idx, first, n):
        if n == 1:
            part[idx] = first
            return
        x = mesh.cell_centroid[idx]
        ext = x.max(axis=0) - x.min(axis=0)
        ax = int(np.argmax(ext[: mesh.dim]))
        order = idx[np.argsort(x[:, ax], kind="stable")]
        na = n // 2
        cut = int(round(len(idx) * na / n))
        split(order[:cut], first, na)
        split(order[cut:], first + na, n - na)

    split(np.arange(mesh.n_cells), 0, nparts)
    return part


def _layers(mesh: Mesh, seed: np.ndarray, layers: int) -> np.ndarray:
    """The cells within `layers` face-neighbour steps of the seed cells (mask)."""
    nb = mesh.cell_nbrs()
    inside = np.zeros(mesh.n_cells, dtype=bool)
    inside[seed] = True
    front = inside.copy()
    for _ in range(layers):
        cand = nb[front]
        cand = cand[cand >= 0]
        new = np.zeros_like(inside)
        new[cand] = True
        front = new & ~inside
        inside |= new
    return inside


def local_mesh(mesh: Mesh, cells: np.ndarray, halo: np.ndarray, name: str = "part") -> Mesh:
    """The sub-mesh of `cells` (global ids, increasing) with the faces that
    touch them in increasing global order; `halo` marks cells left out of the
    CFL minimum."""
    C = mesh.n_cells
    loc = np.full(C, -1, dtype=np.int64)
    loc[cells] = np.arange(len(cells))
    fc = mesh.face_cells.astype(np.int64)
    L, R = fc[:, 0], fc[:, 1]
    inL = loc[L] >= 0
    inR = (R >= 0) & (loc[np.maximum(R, 0)] >= 0)
    faces = np.nonzero(inL | inR)[0]
    floc = np.full(mesh.n_faces, -1, dtype=np.int64)
    floc[faces] = np.arange(len(faces))
    normal = mesh.face_normal[faces].copy()
    bc = mesh.face_bc[faces].copy()
    both = inL[faces] & inR[faces]
    only_L = inL[faces] & ~inR[faces]
    only_R = ~inL[faces] & inR[faces]
    new_fc = np.full((len(faces), 2), -1, dtype=np.int64)
    new_fc[both, 0] = loc[L[faces][both]]
    new_fc[both, 1] = loc[R[faces][both]]
    new_fc[only_L, 0] = loc[L[faces][only_L]]
    new_fc[only_R, 0] = loc[R[faces][only_R]]
    normal[only_R] *= -1.0                      # out of the remaining cell
    cut = (only_L & (R[faces] >= 0)) | only_R   # a neighbour outside the part
    bc[cut] = FACE_NO_CONDITION
    bc[both] = FACE_INTERIOR
    cf = mesh.cell_faces[cells].astype(np.int64)
    cell_faces = np.where(cf >= 0, floc[np.maximum(cf, 0)], -1)
    return Mesh(mesh.dim, mesh.vertices, mesh.cells[cells], mesh.cell_centroid[cells], mesh.cell_volume[cells],
                cell_faces.astype(np.int32), new_fc.astype(np.int32), mesh.face_centroid[faces], normal,
                bc.astype(np.int32), name=name, cell_cfl_skip=halo.astype(np.uint8))


@dataclasses.dataclass
class Part:
    rank: int
    cells: np.ndarray                  # global ids of the local mesh's cells, increasing
    owned: np.ndarray                  # [n_local] bool
    mesh: Mesh
    send: Dict[int, np.ndarray]        # destination part -> local ids of owned cells it needs
    recv: Dict[int, np.ndarray]        # source part -> local ids of halo cells it fills


def build_parts(mesh: Mesh, nparts: int, layers: int, part_of: Optional[np.ndarray] = None) -> List[Part]:
    """Local meshes and the exchange schedule: part r sends to part s its
    owned cells in s's halo, in increasing global id, and s receives them
    into the same cells of its own numbering."""
    part_of = partition_cells(mesh, nparts) if part_of is None else np.asarray(part_of)
    parts = []
    for r in range(nparts):
        own = np.nonzero(part_of == r)[0]
        inside = _layers(mesh, own, layers)
        cells = np.nonzero(inside)[0]
        owned = part_of[cells] == r
        parts.append(Part(r, cells, owned, local_mesh(mesh, cells, ~owned, name="part%d" % r), {}, {}))
    for s in parts:
        halo_g = s.cells[~s.owned]
        for r in range(nparts):
            if r == s.rank:
                continue
            g = halo_g[part_of[halo_g] == r]          # increasing
            if not len(g):
                continue
            rp = parts[r]
            s.recv[r] = np.searchsorted(s.cells, g).astype(np.int32)
            rp.send[s.rank] = np.searchsorted(rp.cells, g).astype(np.int32)
    return parts


class PartitionedSolver:
    """All parts of a partitioned mesh in one process (one device): each part
    an ordinary solver handle, the global dt the minimum of the parts' CFL
    dts, the halo refreshed after every step."""

    def __init__(self, model, mesh: Mesh, settings, params, nparts: int, device: int = 0,
                 part_of: Optional[np.ndarray] = None):
        from .solver import Solver

        self.mesh = mesh
        self.layers = halo_layers(settings.reconstruction_order, settings.ssp_stages)
        self.parts = build_parts(mesh, nparts, self.layers, part_of)
        self.solvers = [Solver(model, p.mesh, settings, params, device=device) for p in self.parts]
        self.nq = self.solvers[0].nq

    def set_state(self, q: np.ndarray, t: float = 0.0):
        for p, s in zip(self.parts, self.solvers):
            s.set_state(q[p.cells], t)

    def dt(self) -> float:
        return min(s.time()[1] for s in self.solvers)

    def time(self) -> float:
        return self.solvers[0].time()[0]

    def exchange(self):
        for p, s in zip(self.parts, self.solvers):
            for dst, cells in p.send.items():
                q = s.get_cells(cells)
                self.solvers[dst].set_cells(self.parts[dst].recv[p.rank], q)

    def step(self, n: int = 1):
        for _ in range(n):
            dt = self.dt()
            for s in self.solvers:
                s.step(1, dts=np.array([dt]))
            self.exchange()

    def get_state(self) -> np.ndarray:
        out = np.empty((self.mesh.n_cells, self.nq))
        for p, s in zip(self.parts, self.solvers):
            q = s.get_state()
            out[p.cells[p.owned]] = q[p.owned]
        return out


def exchange(part: Part, nq: int, get_cells, set_cells, dist, device=None):
    """One halo refresh for this rank's part over torch.distributed:
    get_cells(local ids) gives the owned values ([n, nq]) the schedule sends,
    set_cells(local ids, values) writes the halo cells received.  All sends
    and receives are posted before any is waited on, so no pair of ranks
    depends on the other's order."""
    import torch

    keep, recv, reqs = [], {}, []
    for dst, cells in sorted(part.send.items()):
        v = get_cells(cells)
        buf = v if isinstance(v, torch.Tensor) else torch.as_tensor(np.ascontiguousarray(v, dtype=np.float64))
        buf = buf.to(device) if device is not None else buf
        keep.append(buf)
        reqs.append(dist.isend(buf.contiguous(), dst))
    for src, cells in sorted(part.recv.items()):
        buf = torch.empty((len(cells), nq), dtype=torch.float64, device=device)
        recv[src] = buf
        reqs.append(dist.irecv(buf, src))
    for r in reqs:
        r.wait()
    for src, buf in sorted(recv.items()):
        set_cells(part.recv[src], buf)


def global_dt(local_dt: float, dist, device=None) -> float:
    """The step's dt: the minimum of the parts' CFL dts."""
    import torch

    t = torch.tensor([local_dt], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MIN)
    return float(t.item())


# --------------------------------------------------------------- device form
class TorchComm:
    """The collectives of PartRunner over torch.distributed (NCCL for GPU
    tensors, gloo for CPU tensors).  `stream`: the torch stream the tensors
    are ordered on (the solver handle's), made current while the
    collectives are issued, so NCCL's work is ordered against the handle's
    kernels on the device."""

    def __init__(self, dist, stream=None):
        self.dist = dist
        self.stream = stream

    def _ctx(self):
        import contextlib

        import torch

        return torch.cuda.stream(self.stream) if self.stream is not None else contextlib.nullcontext()

    def min_(self, t):
        with self._ctx():
            self.dist.all_reduce(t, op=self.dist.ReduceOp.MIN)

    def exchange(self, sends, recvs):
        """Post every send and receive, then wait for all: no pair of ranks
        depends on the other's order."""
        with self._ctx():
            ops = [self.dist.P2POp(self.dist.isend, buf, dst) for dst, buf in sorted(sends.items())]
            ops += [self.dist.P2POp(self.dist.irecv, buf, src) for src, buf in sorted(recvs.items())]
            if ops:
                for r in self.dist.batch_isend_irecv(ops):
                    r.wait()


class PartRunner:
    """One part's step loop with the halo refresh.  backend: local_dt()
    -> 1-element tensor of the part's CFL dt; step(dt) at a 1-element tensor
    dt; pack(dst) -> [n, nq] tensor of the owned cells `dst` needs;
    unpack(src, values) into the halo cells `src` fills; recv_buffer(src)
    -> the tensor a message from src lands in.  comm: min_(tensor) in place
    over all parts, exchange(sends, recvs)."""

    def __init__(self, part: Part, backend, comm):
        self.part, self.backend, self.comm = part, backend, comm

    def step(self, n: int = 1):
        for _ in range(n):
            dt = self.backend.local_dt()
            self.comm.min_(dt)
            self.backend.step(dt)
            sends = {dst: self.backend.pack(dst) for dst in self.part.send}
            recvs = {src: self.backend.recv_buffer(src) for src in self.part.recv}
            self.comm.exchange(sends, recvs)
            for src, buf in recvs.items():
                self.backend.unpack(src, buf)


class DevicePart:
    """A part on a GPU: its solver handle and device-resident halo buffers.
    Every call is ordered on the handle's stream (``stream``)."""

    def __init__(self, part: Part, model, settings, params, device: int = 0, launch=None):
        import torch

        from .solver import Solver, set_launch

        self.part = part
        self.solver = Solver(model, part.mesh, settings, params, device=device)
        if launch:
            set_launch(self.solver.h, launch)
        self.lib = self.solver.lib
        self.nq = self.solver.nq
        self.dev = torch.device("cuda", device)
        self.stream = torch.cuda.ExternalStream(self.solver.stream, device=self.dev)
        i32 = dict(dtype=torch.int32, device=self.dev)
        f64 = dict(dtype=torch.float64, device=self.dev)
        # caller (local mesh) ids of the cells each message carries
        self.send_ids = {d: torch.as_tensor(c, **i32) for d, c in part.send.items()}
        self.recv_ids = {s: torch.as_tensor(c, **i32) for s, c in part.recv.items()}
        self.send_buf = {d: torch.empty((len(c), self.nq), **f64) for d, c in part.send.items()}
        self.recv_buf = {s: torch.empty((len(c), self.nq), **f64) for s, c in part.recv.items()}
        self.t_dev = torch.zeros(1, **f64)
        self.dt_dev = torch.zeros(1, **f64)

    def set_state(self, q_global: np.ndarray, t: float = 0.0):
        self.solver.set_state(q_global[self.part.cells], t)

    def local_dt(self):
        from . import native

        native.check(self.lib.zsme_get_time_device(self.solver.h, None, self.dt_dev.data_ptr()))
        return self.dt_dev

    def step(self, dt):
        from . import native

        native.check(self.lib.zsme_step_dt_device(self.solver.h, 1, dt.data_ptr()))

    def pack(self, dst):
        from . import native

        ids, buf = self.send_ids[dst], self.send_buf[dst]
        native.check(self.lib.zsme_get_cells(self.solver.h, len(ids), ids.data_ptr(), buf.data_ptr(), 1))
        return buf

    def recv_buffer(self, src):
        return self.recv_buf[src]

    def unpack(self, src, buf):
        from . import native

        ids = self.recv_ids[src]
        native.check(self.lib.zsme_set_cells(self.solver.h, len(ids), ids.data_ptr(), buf.data_ptr(), 1))

    def owned_state(self):
        """(global ids, values) of the part's owned cells."""
        q = self.solver.get_state()
        return self.part.cells[self.part.owned], q[self.part.owned]


class LocalComm:
    """PartRunner's collectives for several parts held by one process: the
    minimum over the parts' dt tensors, and each packed halo copied into the
    receiving part's buffer.  Parts on one device with their own streams are
    ordered by synchronising the device between the phases (a test and
    single-process harness; across ranks TorchComm keeps everything on the
    device)."""

    def __init__(self):
        self.runners: List[PartRunner] = []
        self._dts = {}
        self._sends = {}

    @staticmethod
    def _sync():
        try:
            import torch

            if torch.cuda.is_available():
                torch.cuda.synchronize()
        except ImportError:
            pass

    def step(self, n: int = 1):
        """Advance every registered part n steps (the per-part PartRunner
        loop, phase by phase across the parts)."""
        for _ in range(n):
            dts = [r.backend.local_dt() for r in self.runners]
            self._sync()
            m = dts[0].clone()
            for d in dts[1:]:
                m = m.minimum(d.to(m.device))
            for d in dts:
                d.copy_(m.to(d.device))
            self._sync()
            for r in self.runners:
                r.backend.step(dts[self.runners.index(r)])
            packed = {(r.part.rank, dst): r.backend.pack(dst) for r in self.runners for dst in r.part.send}
            self._sync()
            by_rank = {r.part.rank: r for r in self.runners}
            for (src, dst), buf in packed.items():
                by_rank[dst].backend.recv_buffer(src).copy_(buf)
            self._sync()
            for r in self.runners:
                for src in r.part.recv:
                    r.backend.unpack(src, r.backend.recv_buffer(src))
            self._sync()
