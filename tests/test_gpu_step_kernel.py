"""Which step kernel a block runs (mplbgpu_step_kernel), and the shifted
forms' interior node pairs on rows shorter than a pair's span: the partner
32 nodes on lies beyond the row (its pulls reach the row padding, the next
rows and, on the last rows of a 2D block, the slack after the last
population) and is computed but never stored, so short rows agree with the
FP64 form as closely as long ones."""
import dataclasses

import numpy as np
import pytest

from mplb_b200 import Solver, config

pytestmark = pytest.mark.gpu


def test_step_kernel_kinds(gpu_lib):
    s = Solver(config.cavity(3, 20, 0.05, re=100))
    assert s.step_kernel(0) == "split"
    s.close()
    s = Solver(dataclasses.replace(config.cavity(3, 8, 0.05, re=100,
                                                 precision="fp32"),
                                   block_sizes=[(2, 9, 9)]))
    assert s.step_kernel(0) == "node"
    s.close()
    s = Solver(config.cavity(3, 12, 0.05, re=100,
                             scheme="Scheme_StreamCollision_Swap"))
    assert s.step_kernel(0) == "swap"
    s.close()


def _run(case, steps):
    with Solver(case) as s:
        s.init_uniform()
        s.stream_collision(steps)
        s.update_macro_vars()
        return [a.copy() for a in s.macro(0)]


@pytest.mark.parametrize("prec,tol", [("fp32", 5e-5), ("fp16", 5e-3)])
@pytest.mark.parametrize("size", [(3, 3), (5, 9), (7, 4), (31, 17), (33, 6),
                                  (3, 3, 3), (9, 5, 4), (35, 7, 3)])
def test_short_rows_close_to_fp64(gpu_lib, size, prec, tol):
    dim = len(size)
    mk = lambda p: dataclasses.replace(
        config.cavity(dim, 8, 0.05, re=100, precision=p), block_sizes=[size])
    # a block of one interior node is not a stable flow: its FP64 and FP32
    # runs part after a few hundred steps (both forms alike), so it is
    # compared over a few steps
    steps = 5 if max(size) == 3 else 300
    ref = _run(mk("fp64"), steps)
    got = _run(mk(prec), steps)
    for a in got:
        assert np.isfinite(a).all()
    speed = np.sqrt(sum(r ** 2 for r in ref[1:]))
    speed_p = np.sqrt(sum(g ** 2 for g in got[1:]))
    assert np.linalg.norm(speed_p - speed) <= tol * np.linalg.norm(speed)
    assert np.linalg.norm(got[0] - ref[0]) <= tol * np.linalg.norm(ref[0])
