"""Slab decomposition of one block (no GPU): slab ranges, the slabs' cases
(cut faces, boundary conditions kept by the end slabs) and the face
exchange between torch.distributed ranks, run as gloo ranks on CPU with
stand-in slabs whose exports are known patterns."""
import os
import socket

import pytest
import torch
import torch.multiprocessing as mp

from mplb_b200 import abi, config, slab


def test_slab_bounds_cover_and_balance():
    for n, parts in ((12, 3), (13, 3), (256, 8), (7, 3), (4, 2)):
        b = slab.slab_bounds(n, parts)
        assert b[0][0] == 0 and b[-1][1] == n
        assert all(b[k][1] == b[k + 1][0] for k in range(parts - 1))
        sizes = [hi - lo for lo, hi in b]
        assert max(sizes) - min(sizes) <= 1 and min(sizes) >= 2
    with pytest.raises(ValueError):
        slab.slab_bounds(5, 3)


def test_slab_cases_keep_end_boundaries_and_cut_the_rest():
    case = config.cavity(3, 12, 0.05, re=100)
    surf = {k: v for k, v in abi.SURFACES.items()}
    cuts, bcs, sizes = [], [], []
    for k in range(3):
        s = slab.slab_case(case, 3, k)
        cuts.append(s.cuts[0])
        bcs.append({b.surface for b in s.boundaries})
        sizes.append(s.block_sizes[0])
    assert cuts == [1 << surf["Front"], (1 << surf["Front"]) |
                    (1 << surf["Back"]), 1 << surf["Back"]]
    side = {"Left", "Right", "Top", "Bottom"}
    assert bcs == [side | {"Back"}, side, side | {"Front"}]
    assert [s[2] for s in sizes] == [4, 4, 4]
    # the lid (Front) boundary keeps its wall velocity in the last slab
    last = slab.slab_case(case, 3, 2)
    lid = [b for b in last.boundaries if b.surface == "Front"][0]
    assert lid.given[0] > 0
    # 2D: slabs along y
    c2 = config.cavity(2, 10, 0.05, re=100)
    s0 = slab.slab_case(c2, 2, 0)
    assert s0.block_sizes[0] == (10, 5)
    assert s0.cuts[0] == 1 << surf["Top"]
    assert "Top" not in {b.surface for b in s0.boundaries}


def test_slab_rejects_connections_and_swap():
    with pytest.raises(ValueError):
        slab.slab_case(config.lchannel(leg=9, side=6, depth=4), 2, 0)
    with pytest.raises(ValueError):
        slab.slab_case(config.cavity(3, 9, 0.05, re=100,
                                     scheme="Scheme_StreamCollision_Swap"),
                       2, 0)


class _FakePart:
    """A slab whose export of side s is filled with (rank, s) and whose
    imports are recorded."""

    def __init__(self, rank, world, nbytes=64):
        self.rank = rank
        self.out, self.inb, self.got = {}, {}, {}
        self.events = []
        for side, present in (("low", rank > 0), ("high", rank < world - 1)):
            self.out[side] = (torch.full((nbytes,), 10 * rank + (side == "high"),
                                         dtype=torch.uint8)
                              if present else None)
            self.inb[side] = (torch.zeros(nbytes, dtype=torch.uint8)
                              if present else None)

    def export_faces(self):
        self.events.append("export")

    def synchronize(self):
        pass

    def step_begin(self):
        self.events.append("begin")

    def step_finish(self):
        self.events.append("finish")

    def import_face(self, side, buf):
        self.got[side] = int(buf[0])
        self.events.append("import")


class _FakeSolver:
    def __init__(self, rank, world):
        self.parts = [_FakePart(rank, world)]
        self.index0 = rank
        self.nparts = world


def _rank(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    s = _FakeSolver(rank, world)
    slab.DistExchange().step(s)
    out.put((rank, dict(s.parts[0].got), list(s.parts[0].events)))
    dist.barrier()
    dist.destroy_process_group()


def test_faces_cross_between_three_gloo_ranks():
    """Rank k's low halo gets rank k-1's high export and its high halo
    rank k+1's low export, after its step's interior part was queued and
    before the step is finished."""
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    world = 3
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q))
             for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    got = {r: g for r, g, _ in res}
    events = {r: e for r, _, e in res}
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    # the faces move between the step's interior part and its finish
    nimp = {0: 1, 1: 2, 2: 1}
    for r in range(world):
        assert events[r] == ["export", "begin"] + ["import"] * nimp[r] + \
            ["finish"]
    assert got[0] == {"high": 10 * 1 + 0}
    assert got[1] == {"low": 10 * 0 + 1, "high": 10 * 2 + 0}
    assert got[2] == {"low": 10 * 1 + 1}
