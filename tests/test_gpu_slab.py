"""A block decomposed into slabs (cut faces, face exchange before every
step) against the same block in one piece, on one GPU: the slabs are
contexts of this process and the faces move by device copies
(LocalExchange).  FP64 and FP32 results are bit for bit those of the whole
block; residuals (summed per slab, then added) within 1e-12."""
import numpy as np
import pytest

from mplb_b200 import Solver, abi, config, slab
from mplb_b200.solver import MplbGpuError

pytestmark = pytest.mark.gpu


def whole_and_slabs(case, parts, steps, check=None):
    w = Solver(case)
    w.init_uniform()
    s = slab.SlabSolver(case, parts, list(range(parts)), slab.LocalExchange())
    s.init_uniform()
    for k in steps:
        w.stream_collision(k)
        s.stream_collision(k)
        assert np.array_equal(s.f(), w.f(0)), k
        w.update_macro_vars()
        s.update_macro_vars()
        for a, b in zip(s.macro(), w.macro(0)):
            assert np.array_equal(a, b), k
        if check:
            rw = w.calc_residual_error(check)
            rs = s.calc_residual_error(check)
            np.testing.assert_allclose(rs[1], rw[1], rtol=1e-12)
            np.testing.assert_allclose(rs[0], rw[0], rtol=1e-12)
    w.close()
    s.close()


@pytest.mark.parametrize("parts", [2, 3])
def test_cavity3d_slabs_match_whole_block(gpu_lib, parts):
    whole_and_slabs(config.cavity(3, 20, 0.05, re=100), parts, [1, 1, 5, 13],
                    check=20)


def test_cavity3d_fp32_slabs_match_whole_block(gpu_lib):
    whole_and_slabs(config.cavity(3, 18, 0.05, re=100, precision="fp32"), 2,
                    [1, 7, 12])


def test_cavity3d_bounce_back_uneven_slabs(gpu_lib):
    case = config.cavity(3, 17, 0.05, re=100, wall="HalfwayBounceBack")
    whole_and_slabs(case, 4, [3, 9])


def test_cavity2d_slabs_match_whole_block(gpu_lib):
    whole_and_slabs(config.cavity(2, 33, 0.05, re=100), 3, [1, 10, 40],
                    check=51)


def test_cut_faces_are_checked(gpu_lib):
    case = config.cavity(3, 10, 0.05, re=100)
    bad = slab.slab_case(case, 2, 0)
    bad.boundaries = list(case.boundaries)     # a wall on the cut face
    with pytest.raises(MplbGpuError) as e:
        Solver(bad)
    assert e.value.status == abi.ERR_INVALID
    s = Solver(slab.slab_case(case, 2, 0))
    s.init_uniform()
    buf = np.zeros(4)
    rc = s.lib.mplbgpu_export_face(s.h, 0, abi.SURFACES["Back"],
                                   buf.ctypes.data)
    assert rc == abi.ERR_INVALID      # Back is a wall here, not a cut
    s.close()


def _slab_rank(rank, world, port, steps, out):
    import os

    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    torch.cuda.set_device(0)
    case = config.cavity(3, 16, 0.05, re=100)
    s = slab.SlabSolver(case, world, [rank], slab.DistExchange())
    s.init_uniform()
    s.stream_collision(steps)
    s.update_macro_vars()

    def reduce(d, t):
        dt = torch.tensor(np.concatenate([d, t]))
        dist.all_reduce(dt)
        v = dt.numpy()
        return v[:len(d)], v[len(d):]

    res = s.calc_residual_error(10, reduce=reduce)
    out.put((rank, s.f(), res[0]))
    dist.barrier()
    s.close()
    dist.destroy_process_group()


def test_slab_ranks_through_torch_distributed(gpu_lib):
    """Two processes, one slab each, faces exchanged by DistExchange (gloo,
    staged through host memory: both ranks share this GPU, so no kernel
    waits on the other rank)."""
    import socket

    import torch.multiprocessing as mp
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    steps, world = 23, 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_slab_rank, args=(r, world, port, steps, q))
             for r in range(world)]
    for p in procs:
        p.start()
    got = {}
    for _ in range(world):
        rank, f, res = q.get(timeout=300)
        got[rank] = (f, res)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    w = Solver(config.cavity(3, 16, 0.05, re=100))
    w.init_uniform()
    w.stream_collision(steps)
    w.update_macro_vars()
    rw = w.calc_residual_error(10)
    assert np.array_equal(np.concatenate([got[0][0], got[1][0]], axis=0),
                          w.f(0))
    np.testing.assert_allclose(got[0][1], rw[0], rtol=1e-12)
    w.close()


def test_slab_checkpoint_round_trips_with_the_whole_block(gpu_lib, tmp_path):
    """Slabs checkpoint into the whole block's files and restart from them
    either way, bit for bit the uninterrupted whole-block run."""
    from mplb_b200 import checkpoint
    case = config.cavity(3, 18, 0.05, re=100)
    w = Solver(case)
    w.init_uniform()
    w.stream_collision(21)
    want = w.f(0)
    w.close()
    s = slab.SlabSolver(case, 3, [0, 1, 2], slab.LocalExchange())
    s.init_uniform()
    s.stream_collision(7)
    checkpoint.save_slabs(s, str(tmp_path), 7)
    s.close()
    r = checkpoint.restart(case, str(tmp_path), 7)      # as the whole block
    r.stream_collision(7)
    checkpoint.save(r, str(tmp_path), 14)
    r.close()
    s2 = checkpoint.restart_slabs(case, 2, str(tmp_path), 14)   # as 2 slabs
    s2.stream_collision(7)
    assert np.array_equal(s2.f(), want)
    s2.close()
