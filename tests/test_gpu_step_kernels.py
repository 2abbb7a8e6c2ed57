"""The two launch layouts of the fused step give the same bits: the
one-launch split kernel (boundary-shell rows, x faces, interior warp tasks)
and the default edge + software-pipelined interior pair
(MPLB_B200_STEP_KERNEL=split selects the former at context creation).
FP64 and FP32 compute every node the same way in both, so f and the
moments agree bit for bit; FP16 pairs its nodes differently for the
stochastic rounding draws, so its two layouts agree to its rounding."""
import dataclasses

import numpy as np
import pytest

from mplb_b200 import Solver, config

pytestmark = pytest.mark.gpu


def run(case, steps, layout, monkeypatch):
    if layout == "split":
        monkeypatch.setenv("MPLB_B200_STEP_KERNEL", "split")
    else:
        monkeypatch.delenv("MPLB_B200_STEP_KERNEL", raising=False)
    s = Solver(case)
    s.init_uniform()
    launches0 = s.launch_count()
    s.stream_collision(steps)
    per_step = (s.launch_count() - launches0) / steps
    s.update_macro_vars()
    out = ([s.f(b) for b in case.block_ids],
           [s.macro(b) for b in case.block_ids], per_step)
    s.close()
    return out


CASES = {
    "cavity3d_40": lambda p: config.cavity(3, 40, 0.05, re=400, precision=p),
    # rows of 37 / 70 nodes: pipelined tasks end inside a row
    "box3d_70x9x11": lambda p: dataclasses.replace(
        config.cavity(3, 8, 0.05, re=200, precision=p),
        block_sizes=[(70, 9, 11)]),
    "box3d_37x12x6": lambda p: dataclasses.replace(
        config.cavity(3, 8, 0.05, re=200, precision=p),
        block_sizes=[(37, 12, 6)]),
    "cavity2d_100": lambda p: config.cavity(2, 100, 0.05, re=400, precision=p),
    "poiseuille3d": lambda p: config.poiseuille(3, 48, 20, 12,
                                                g_lattice=1e-5, precision=p),
    "lchannel": lambda p: config.lchannel(leg=64, side=24, depth=12,
                                          precision=p),
}


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
@pytest.mark.parametrize("name", sorted(CASES))
def test_layouts_bitwise(gpu_lib, monkeypatch, name, prec):
    case = CASES[name](prec)
    f_s, m_s, n_s = run(case, 30, "split", monkeypatch)
    f_p, m_p, n_p = run(case, 30, "pipe", monkeypatch)
    for a, b in zip(f_s, f_p):
        assert np.array_equal(a, b)
    for ma, mb in zip(m_s, m_p):
        for a, b in zip(ma, mb):
            assert np.array_equal(a, b)
    # the pipelined layout is two launches per block and step
    assert n_p >= n_s


def test_layouts_fp16_close(gpu_lib, monkeypatch):
    case = config.cavity(3, 40, 0.05, re=400, precision="fp16")
    _, m_s, _ = run(case, 30, "split", monkeypatch)
    _, m_p, _ = run(case, 30, "pipe", monkeypatch)
    u_s, u_p = m_s[0][1], m_p[0][1]
    assert np.linalg.norm(u_s - u_p) / np.linalg.norm(u_s) < 1e-2


@pytest.mark.parametrize("name", ["cavity3d_40", "lchannel", "cavity2d_100"])
def test_step_in_two_parts_is_one_step(gpu_lib, monkeypatch, name):
    """mplbgpu_step_begin + mplbgpu_step_finish is one mplbgpu_step, bit
    for bit (FP64; single block, three joined blocks with halos and a
    pressure outlet, 2D)."""
    from mplb_b200 import abi
    monkeypatch.delenv("MPLB_B200_STEP_KERNEL", raising=False)
    case = CASES[name]("fp64")
    a = Solver(case)
    a.init_uniform()
    a.stream_collision(12)
    b = Solver(case)
    b.init_uniform()
    lib = b.lib
    for _ in range(12):
        assert lib.mplbgpu_step_begin(b.h) == abi.OK
        assert lib.mplbgpu_step_finish(b.h) == abi.OK
    for blk in case.block_ids:
        assert np.array_equal(a.f(blk), b.f(blk))
    a.close()
    b.close()


def test_step_in_two_parts_state_errors(gpu_lib):
    from mplb_b200 import abi
    case = config.cavity(3, 20, 0.05, re=100)
    s = Solver(case)
    s.init_uniform()
    lib = s.lib
    assert lib.mplbgpu_step_finish(s.h) == abi.ERR_STATE
    assert lib.mplbgpu_step_begin(s.h) == abi.OK
    assert lib.mplbgpu_step_begin(s.h) == abi.ERR_STATE
    assert lib.mplbgpu_step(s.h, 1) == abi.ERR_STATE
    assert lib.mplbgpu_update_macro(s.h) == abi.ERR_STATE
    assert lib.mplbgpu_step_finish(s.h) == abi.OK
    assert lib.mplbgpu_step(s.h, 1) == abi.OK
    s.close()
    sw = Solver(config.cavity(3, 12, 0.05, re=100,
                              scheme="Scheme_StreamCollision_Swap"))
    sw.init_uniform()
    assert sw.lib.mplbgpu_step_begin(sw.h) == abi.ERR_UNSUPPORTED
    sw.close()
