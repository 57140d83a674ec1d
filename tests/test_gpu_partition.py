"""The partitioned GPU step (zoomy-dmplex_b200/partition.py): every part an
ordinary solver handle on its local mesh, the halo refreshed through
zsme_get_cells / zsme_set_cells after each step, the dt the minimum over the
parts -- against the undivided GPU run, bit for bit."""
import numpy as np
import pytest

from zoomy_dmplex_b200 import cases, partition as P
from zoomy_dmplex_b200.solver import Solver

from test_gpu_parity import params

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,nparts", [("l2", 2), ("l2", 4), ("l4", 3), ("mixed", 3)])
def test_partitioned_equals_undivided(name, nparts):
    c = {"l2": lambda: cases.level2(40), "l4": lambda: cases.roofline_l4(36),
         "mixed": lambda: cases.mixed_level2(30)}[name]()
    p = params(c.model, c.params)
    g = Solver(c.model, c.mesh, c.settings, p)
    g.set_state(c.q0)
    ps = P.PartitionedSolver(c.model, c.mesh, c.settings, p, nparts)
    ps.set_state(c.q0)
    assert ps.dt() == g.time()[1]
    for k in range(20):
        g.step(1)
        ps.step(1)
    assert ps.time() == g.time()[0]
    assert np.array_equal(ps.get_state(), g.get_state())


def test_cells_io_round_trip():
    c = cases.level2(20)
    g = Solver(c.model, c.mesh, c.settings, params(c.model, c.params))
    g.set_state(c.q0)
    ids = np.array([5, 0, 17, 3], dtype=np.int32)
    assert np.array_equal(g.get_cells(ids), g.get_state()[ids])
    q = g.get_state()
    new = q[ids] * 1.01
    g.set_cells(ids, new)
    q[ids] = new
    assert np.array_equal(g.get_state(), q)
    a = g.get_aux()
    g.set_state(q)                       # aux recomputed from the same state
    assert np.array_equal(g.get_aux()[ids], a[ids])


@pytest.mark.parametrize("nparts,mixed", [(2, False), (3, True)])
def test_device_parts_equal_undivided(nparts, mixed):
    """The device-resident form: DevicePart handles on this GPU, the dt read
    and imposed in device memory (zsme_get_time_device / zsme_step_dt_device),
    halos packed and unpacked by zsme_get_cells / zsme_set_cells on device
    buffers and copied part to part (LocalComm); 20 steps bit-identical to
    the undivided GPU run."""
    c = cases.mixed_level2(18) if mixed else cases.level2(40)
    p = params(c.model, c.params)
    steps = 20
    g = Solver(c.model, c.mesh, c.settings, p)
    g.set_state(c.q0)
    g.step(steps)
    full = g.get_state()
    parts = P.build_parts(c.mesh, nparts, P.halo_layers(2, c.settings.ssp_stages))
    comm = P.LocalComm()
    devs = []
    for pt in parts:
        d = P.DevicePart(pt, c.model, c.settings, p)
        d.set_state(c.q0)
        devs.append(d)
        comm.runners.append(P.PartRunner(pt, d, comm))
    comm.step(steps)
    got = np.full_like(full, np.nan)
    for d in devs:
        cells, vals = d.owned_state()
        got[cells] = vals
        assert d.solver.time()[0] == g.time()[0]
    assert np.array_equal(got, full)


def _nccl_one_rank(port, q):
    import os

    import torch
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", rank=0, world_size=1)
    try:
        c = cases.level2(30)
        p = params(c.model, c.params)
        parts = P.build_parts(c.mesh, 1, P.halo_layers(2, c.settings.ssp_stages))
        d = P.DevicePart(parts[0], c.model, c.settings, p)
        d.set_state(c.q0)
        P.PartRunner(parts[0], d, P.TorchComm(dist, d.stream)).step(10)
        g = Solver(c.model, c.mesh, c.settings, p)
        g.set_state(c.q0)
        g.step(10)
        cells, vals = d.owned_state()
        q.put(bool(np.array_equal(vals, g.get_state()[cells])) and d.solver.time() == g.time())
    finally:
        dist.destroy_process_group()


def test_nccl_runner_one_rank():
    """TorchComm over NCCL on the handle's stream with one rank (this run has
    one GPU): the device all-reduce of the dt and the stream-ordered step
    reproduce the plain run bit for bit."""
    import multiprocessing as mp
    import socket

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    pr = ctx.Process(target=_nccl_one_rank, args=(port, q))
    pr.start()
    ok = q.get(timeout=300)
    pr.join(timeout=60)
    assert ok and pr.exitcode == 0
