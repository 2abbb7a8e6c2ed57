"""The shifted forms' split step with its interior tiles loaded by TMA
(SplitTmaStepKernel) gives the per-thread-load split step's results bit for
bit: same node pairs, same arithmetic, same FP16 rounding draws.  Cases
cover row counts that are not a multiple of the tile's 4 rows, row lengths
that are not a multiple of its 64 columns, 2D, a body force, joined blocks
with a pressure outlet, and the step in two parts."""
import dataclasses
import os

import numpy as np
import pytest

from mplb_b200 import Solver, config

pytestmark = pytest.mark.gpu

CASES = {
    "cavity3d_40": lambda p: config.cavity(3, 40, 0.05, re=400, precision=p),
    "box3d_37x14x6": lambda p: dataclasses.replace(
        config.cavity(3, 8, 0.05, re=200, precision=p),
        block_sizes=[(37, 14, 6)]),
    "box3d_130x9x5": lambda p: dataclasses.replace(
        config.cavity(3, 8, 0.05, re=200, precision=p),
        block_sizes=[(130, 9, 5)]),
    "box3d_3x3x3": lambda p: dataclasses.replace(
        config.cavity(3, 8, 0.05, re=200, precision=p),
        block_sizes=[(3, 3, 3)]),
    "cavity2d_100": lambda p: config.cavity(2, 100, 0.05, re=400, precision=p),
    "box2d_70x13": lambda p: dataclasses.replace(
        config.cavity(2, 8, 0.05, re=200, precision=p),
        block_sizes=[(70, 13)]),
    "poiseuille3d": lambda p: config.poiseuille(3, 48, 21, 11,
                                                g_lattice=1e-5, precision=p),
    "lchannel": lambda p: config.lchannel(leg=64, side=22, depth=13,
                                          precision=p),
}


def _solver(case, tma):
    old = os.environ.get("MPLBGPU_NO_TMA")
    try:
        if tma:
            os.environ.pop("MPLBGPU_NO_TMA", None)
        else:
            os.environ["MPLBGPU_NO_TMA"] = "1"
        s = Solver(case)
    finally:
        if old is None:
            os.environ.pop("MPLBGPU_NO_TMA", None)
        else:
            os.environ["MPLBGPU_NO_TMA"] = old
    return s


@pytest.mark.parametrize("prec", ["fp32", "fp16"])
@pytest.mark.parametrize("name", sorted(CASES))
def test_tma_interior_matches_per_thread_loads(gpu_lib, name, prec):
    case = CASES[name](prec)
    a = _solver(case, tma=False)
    b = _solver(case, tma=True)
    kinds = {blk: b.step_kernel(blk) for blk in case.block_ids}
    assert all(a.step_kernel(blk) != "split_tma" for blk in case.block_ids)
    if name != "box3d_3x3x3":   # a box wider than the block may be refused
        assert any(k == "split_tma" for k in kinds.values()), kinds
    for s in (a, b):
        s.init_uniform()
        s.stream_collision(15)
    for blk in case.block_ids:
        fa, fb = a.f(blk), b.f(blk)
        assert np.isfinite(fa).all()
        assert np.array_equal(fa, fb), (blk, np.abs(fa - fb).max())
    a.close()
    b.close()


@pytest.mark.parametrize("prec", ["fp32", "fp16"])
def test_tma_step_in_two_parts(gpu_lib, prec):
    case = dataclasses.replace(config.cavity(3, 8, 0.05, re=200,
                                             precision=prec),
                               block_sizes=[(67, 18, 9)])
    a = _solver(case, tma=True)
    b = _solver(case, tma=True)
    for s in (a, b):
        s.init_uniform()
    a.stream_collision(10)
    for _ in range(10):
        assert b.lib.mplbgpu_step_begin(b.h) == 0
        assert b.lib.mplbgpu_step_finish(b.h) == 0
    assert np.array_equal(a.f(0), b.f(0))
    a.close()
    b.close()


def test_fp64_keeps_the_split_step(gpu_lib):
    s = Solver(config.cavity(3, 20, 0.05, re=100))
    assert s.step_kernel(0) == "split"
    s.close()
    s = Solver(dataclasses.replace(config.cavity(3, 8, 0.05, re=100,
                                                 precision="fp32"),
                                   block_sizes=[(2, 9, 9)]))
    assert s.step_kernel(0) == "node"
    s.close()
