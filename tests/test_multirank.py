"""The multi-rank paths on CPU with the gloo backend, world size 2:
the ensemble's instance shards (greedy balance on cell counts) are disjoint,
cover every instance and balance the ranks' cells, as every rank computes
them on its own; the bench's timing reduction (max over ranks) and its
per-rank replica accounting hold."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, n_total, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        from zoomy_dmplex_b200 import cases

        shard = cases.ensemble_shard(n_total, world, rank)
        cells = sum(2 * (cases.ensemble_side(i) - 1) ** 2 for i in shard)
        shards = [None] * world
        dist.all_gather_object(shards, (shard, cells))
        ms = torch.tensor([10.0 + rank], dtype=torch.float64)
        dist.all_reduce(ms, op=dist.ReduceOp.MAX)
        if rank == 0:
            q.put((shards, float(ms.item())))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("n_total", [64, 512])
def test_ensemble_shards_two_ranks(n_total):
    from zoomy_dmplex_b200 import cases

    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    mp.start_processes(_worker, args=(world, _free_port(), n_total, q), nprocs=world, join=True,
                       start_method="spawn")
    shards, ms_max = q.get()
    idx = sorted(i for s, _ in shards for i in s)
    assert idx == list(range(n_total))                       # disjoint and complete
    loads = [c for _, c in shards]
    assert max(loads) / min(loads) < 1.01                    # balanced cells
    assert shards[0][0] == cases.ensemble_shard(n_total, world, 0)  # same answer on every rank
    assert ms_max == 11.0                                    # max over ranks


def test_shard_instances_greedy():
    from zoomy_dmplex_b200 import cases

    sh = cases.shard_instances([5, 9, 1, 4, 4, 3], 2)
    assert sorted(sh[0] + sh[1]) == list(range(6))
    loads = [sum([5, 9, 1, 4, 4, 3][i] for i in s) for s in sh]
    assert abs(loads[0] - loads[1]) <= 1
