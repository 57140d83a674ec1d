"""Spatial partition with halo exchange (zoomy-dmplex_b200/partition.py).

* the parts' owned cells cover the mesh once, halos are the 2 s cell layers
  an order-2 SSP-RK(s,2) step reads, and the exchange schedule matches send
  and receive lists cell for cell;
* the partitioned step run on oracles (one per part, halo refreshed through
  the oracles' states after every step, dt = minimum over the parts) equals
  the undivided oracle run bit for bit -- the local meshes, the halo depth,
  the CFL mask of halo cells and the dt reduction together;
* two gloo ranks exchange their halos with torch.distributed.
"""
import multiprocessing as mp
import os
import socket

import numpy as np
import pytest

import oracle_py as O
from zoomy_dmplex_b200 import cases, models, partition as P


@pytest.fixture(scope="module", autouse=True)
def _threads():
    O.set_threads(0)


def params(case):
    names, vals = models.parameter_table(case.model)
    for k, v in case.params.items():
        vals[names.index(k)] = v
    return np.array(vals)


@pytest.mark.parametrize("nparts", [2, 3, 4])
def test_parts_cover_and_schedule(nparts):
    m = cases.level2(30).mesh
    layers = P.halo_layers(2, 2)
    assert layers == 4
    parts = P.build_parts(m, nparts, layers)
    owner = np.full(m.n_cells, -1)
    for p in parts:
        g = p.cells[p.owned]
        assert np.all(owner[g] == -1)
        owner[g] = p.rank
        assert np.all(np.diff(p.cells) > 0)
        # the halo is exactly the cells within `layers` steps of the owned ones
        inside = P._layers(m, g, layers)
        assert np.array_equal(np.nonzero(inside)[0], p.cells)
        assert np.array_equal(p.mesh.cell_cfl_skip.astype(bool), ~p.owned)
    assert np.all(owner >= 0)
    sizes = np.bincount(owner, minlength=nparts)
    assert sizes.max() - sizes.min() <= 1
    for s in parts:
        got = np.zeros(len(s.cells), dtype=bool)
        for r, recv in s.recv.items():
            send = parts[r].send[s.rank]
            assert np.array_equal(parts[r].cells[send], s.cells[recv])
            assert np.all(parts[r].owned[send]) and not np.any(s.owned[recv])
            got[recv] = True
        assert np.array_equal(got, ~s.owned)


def _oracle_partitioned(case, nparts, steps):
    m, st, p = case.mesh, case.settings.to_struct(), params(case)
    parts = P.build_parts(m, nparts, P.halo_layers(case.settings.reconstruction_order, case.settings.ssp_stages))
    ors = [O.Oracle(case.model, pt.mesh.as_abi_arrays(), st, p) for pt in parts]
    for pt, o in zip(parts, ors):
        o.set_state(case.q0[pt.cells])
    for _ in range(steps):
        dt = min(o.time()[1] for o in ors)
        for o in ors:
            o.step(1, dts=[dt])
        t = ors[0].time()[0]
        qs = [o.get_state() for o in ors]
        for pt, o in zip(parts, ors):
            for src, recv in pt.recv.items():
                qs[pt.rank][recv] = qs[src][parts[src].send[pt.rank]]
        for pt, o, q in zip(parts, ors, qs):
            o.set_state(q, t)
    out = np.empty_like(case.q0)
    for pt, o in zip(parts, ors):
        out[pt.cells[pt.owned]] = o.get_state()[pt.owned]
    return out, ors[0].time()[0]


@pytest.mark.parametrize("nparts,mixed", [(2, False), (4, False), (3, True)])
def test_partitioned_oracle_equals_undivided(nparts, mixed):
    c = cases.mixed_level2(18) if mixed else cases.level2(24)
    steps = 15
    o = O.Oracle(c.model, c.mesh.as_abi_arrays(), c.settings.to_struct(), params(c))
    o.set_state(c.q0)
    o.step(steps)
    q, t = _oracle_partitioned(c, nparts, steps)
    assert t == o.time()[0]
    assert np.array_equal(q, o.get_state())


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        c = cases.level2(20)
        parts = P.build_parts(c.mesh, world, 4)
        pt = parts[rank]
        local = c.q0[pt.cells].copy()
        local[~pt.owned] = -1.0                          # stale halo

        def get_cells(ids):
            return local[ids]

        def set_cells(ids, vals):
            local[ids] = vals.numpy()

        P.exchange(pt, local.shape[1], get_cells, set_cells, dist)
        ok = bool(np.array_equal(local, c.q0[pt.cells]))
        dt = P.global_dt(0.1 * (rank + 1), dist)
        q.put((rank, ok, dt))
    finally:
        dist.destroy_process_group()


def test_gloo_halo_exchange():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = sorted(q.get(timeout=240) for _ in ps)
    for p in ps:
        p.join(timeout=60)
    assert [r[1] for r in res] == [True, True]
    assert [r[2] for r in res] == [0.1, 0.1]


class OracleBackend:
    """PartRunner's backend over an oracle part (CPU tensors): what
    DevicePart does on the GPU -- the part's CFL dt, a step at an imposed dt,
    owned cells packed for a neighbour, received values unpacked into the
    halo -- on the CPU restatement."""

    def __init__(self, part, oracle, nq):
        self.part, self.o, self.nq = part, oracle, nq

    def local_dt(self):
        import torch

        return torch.tensor([self.o.time()[1]], dtype=torch.float64)

    def step(self, dt):
        self.o.step(1, dts=[float(dt.item())])

    def pack(self, dst):
        import torch

        return torch.from_numpy(np.ascontiguousarray(self.o.get_state()[self.part.send[dst]]))

    def recv_buffer(self, src):
        import torch

        return torch.empty((len(self.part.recv[src]), self.nq), dtype=torch.float64)

    def unpack(self, src, buf):
        q = self.o.get_state()
        q[self.part.recv[src]] = buf.numpy()
        self.o.set_state(q, self.o.time()[0])


def _runner_rank(rank, world, port, q, steps):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        c = cases.level2(24)
        parts = P.build_parts(c.mesh, world, P.halo_layers(2, c.settings.ssp_stages))
        pt = parts[rank]
        o = O.Oracle(c.model, pt.mesh.as_abi_arrays(), c.settings.to_struct(), params(c))
        o.set_state(c.q0[pt.cells])
        P.PartRunner(pt, OracleBackend(pt, o, c.q0.shape[1]), P.TorchComm(dist)).step(steps)
        q.put((rank, pt.cells[pt.owned], o.get_state()[pt.owned], o.time()[0]))
    finally:
        dist.destroy_process_group()


def test_gloo_part_runner_equals_undivided():
    """PartRunner over torch.distributed (two gloo ranks, one oracle part
    each): the global dt by all-reduce MIN, the step, the halo exchange by
    batched point-to-point messages; 12 steps end bit for bit on the
    undivided oracle run."""
    steps = 12
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_runner_rank, args=(r, 2, port, q, steps)) for r in range(2)]
    for p in ps:
        p.start()
    res = [q.get(timeout=300) for _ in ps]
    for p in ps:
        p.join(timeout=60)
    c = cases.level2(24)
    o = O.Oracle(c.model, c.mesh.as_abi_arrays(), c.settings.to_struct(), params(c))
    o.set_state(c.q0)
    o.step(steps)
    full = o.get_state()
    got = np.full_like(full, np.nan)
    for _, cells, vals, t in res:
        got[cells] = vals
        assert t == o.time()[0]
    assert np.array_equal(got, full)
