"""The one-array swap scheme (SchemeType Scheme_StreamCollision_Swap) on the
GPU, through the C ABI.

The golden fixtures made by the reference's own swap step are replayed by
test_gpu_parity.py (bit for bit).  Here the CUDA path is compared with the
oracle (the C restatement of the reference's swap step) after every step
count from 1 to 8 - the in-place kernels alternate between two layouts of
the one array, so odd and even counts read the state differently - and
after a restart from downloaded f, with and without the body force."""
import dataclasses

import numpy as np
import pytest

from mplb_b200 import Solver, abi, config
from mplb_b200.solver import MplbGpuError

pytestmark = pytest.mark.gpu

SWAP = "Scheme_StreamCollision_Swap"


def box(nx, ny, nz, force=False, precision="fp64"):
    c = config.cavity(3, max(nx, ny, nz), 0.05, re=150, scheme=SWAP,
                      precision=precision)
    c = dataclasses.replace(c, block_sizes=[(nx, ny, nz)])
    if force:
        c = dataclasses.replace(c, body_force="BodyForce_1st",
                                accel=(2e-3, -1e-3, 3e-3),
                                force_velocity=True)
    return c


@pytest.mark.parametrize("shape,force", [((13, 11, 9), True),
                                         ((16, 16, 16), False),
                                         ((33, 5, 7), True)])
def test_swap_matches_oracle_every_step(gpu_lib, oracle_mod, shape, force):
    case = box(*shape, force=force)
    o = oracle_mod.Oracle(case)
    o.init_uniform()
    s = Solver(case)
    s.init_uniform()
    assert np.array_equal(s.f(0), o.f(0))
    for step in range(1, 9):
        o.step(1)
        s.stream_collision(1)
        assert np.array_equal(s.f(0), o.f(0)), step
        o.update_macro()
        s.update_macro_vars()
        for got, want in zip(s.macro(0), o.macro(0)):
            assert np.array_equal(got, want), step
    o.step(25)
    s.stream_collision(25)
    assert np.array_equal(s.f(0), o.f(0))
    s.close()


@pytest.mark.parametrize("first", [6, 7])
def test_swap_restart_from_downloaded_f(gpu_lib, first):
    case = box(12, 10, 8, force=True)
    a = Solver(case)
    a.init_uniform()
    a.stream_collision(first)
    saved = a.f(0)
    a.stream_collision(9)
    b = Solver(case)
    b.upload_f(0, saved)
    b.stream_collision(9)
    assert np.array_equal(a.f(0), b.f(0))
    a.update_macro_vars()
    b.update_macro_vars()
    for x, y in zip(a.macro(0), b.macro(0)):
        assert np.array_equal(x, y)


def test_swap_fp32_fp16_close_to_fp64(gpu_lib):
    """The shifted FP32 and FP16-storage forms of the swap step against its
    FP64 form."""
    out = {}
    for prec in ("fp64", "fp32", "fp16"):
        s = Solver(box(24, 24, 24, precision=prec))
        s.init_uniform()
        s.stream_collision(400)
        s.update_macro_vars()
        out[prec] = s.macro(0)
        s.close()
    for k in (1, 3):   # u and w; v is the small cross-flow
        ref = out["fp64"][k]
        for prec, tol in (("fp32", 1e-5), ("fp16", 5e-3)):
            err = np.linalg.norm(out[prec][k] - ref) / np.linalg.norm(ref)
            assert err < tol, (prec, k, err)


def test_swap_rejects_cases_outside_its_scope(gpu_lib):
    bad = [config.cavity(2, 9, 0.05, re=100, scheme=SWAP),
           config.cavity(3, 9, 0.05, re=100, scheme=SWAP,
                         wall="HalfwayBounceBack"),
           dataclasses.replace(config.lchannel(leg=9, side=6, depth=4),
                               scheme=SWAP)]
    for case in bad:
        with pytest.raises(MplbGpuError) as e:
            Solver(case)
        assert e.value.status == abi.ERR_UNSUPPORTED
