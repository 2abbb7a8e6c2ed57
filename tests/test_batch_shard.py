"""Partition of the batched cavities over ranks (no GPU): LPT balance,
determinism, and agreement between two gloo ranks that each compute their
shard independently."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from mplb_b200 import batch


def test_lpt_covers_every_cavity_once_and_balances():
    specs = batch.cavity_set(4096)
    costs = [float(s.n * s.n) for s in specs]
    for world in (1, 2, 3, 8):
        parts = batch.lpt_shards(costs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(specs)))
        loads = [sum(costs[i] for i in p) for p in parts]
        # LPT is within the largest item of the mean
        assert max(loads) - min(loads) <= max(costs)


def test_lpt_is_deterministic_and_order_independent_of_rank():
    costs = [5.0, 3.0, 3.0, 8.0, 1.0, 5.0]
    a = batch.lpt_shards(costs, 2)
    b = batch.lpt_shards(list(costs), 2)
    assert a == b
    # by cost 8 (3), 5 (0), 5 (5), 3 (1), 3 (2), 1 (4), each to the lighter
    assert a == [[1, 3, 4], [0, 2, 5]]


def _rank(rank, world, port, out):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    specs = batch.cavity_set(512)
    mine = batch.shard(specs, rank, world)
    t = torch.zeros(len(specs), dtype=torch.int64)
    t[mine] = 1
    dist.all_reduce(t)
    nodes = torch.tensor([float(sum(specs[i].n ** 2 for i in mine))],
                         dtype=torch.float64)
    allnodes = [torch.zeros(1, dtype=torch.float64) for _ in range(world)]
    dist.all_gather(allnodes, nodes)
    if rank == 0:
        out.put((t.tolist(), [float(x) for x in allnodes]))
    dist.destroy_process_group()


def test_two_gloo_ranks_cover_the_set_exactly_once():
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    cover, loads = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert set(cover) == {1}
    specs = batch.cavity_set(512)
    assert abs(loads[0] - loads[1]) <= max(s.n ** 2 for s in specs)
    assert sum(loads) == sum(s.n ** 2 for s in specs)
