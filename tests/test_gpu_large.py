"""Blocks beyond 2^31 population elements.

Such blocks run kernels with 64-bit element offsets (the usual ones use
32-bit offsets from the node's address).  MPLB_B200_WIDE_OFFSETS=1 selects
the 64-bit kernels for any block, so they are checked bit for bit against
the 32-bit ones on small cases of every kind; then a closed cavity of
1024 x 1024 x 130 nodes (2.6e9 FP64 elements per array) steps with mass
conserved and a healthy state."""
import os

import numpy as np
import pytest

from mplb_b200 import Solver, abi, config

pytestmark = pytest.mark.gpu

WIDE = "MPLB_B200_WIDE_OFFSETS"


def run(case, steps, wide):
    old = os.environ.get(WIDE)
    os.environ[WIDE] = "1" if wide else "0"
    try:
        s = Solver(case)
    finally:
        if old is None:
            del os.environ[WIDE]
        else:
            os.environ[WIDE] = old
    s.init_uniform()
    s.stream_collision(steps)
    s.update_macro_vars()
    out = ([s.f(b) for b in case.block_ids],
           [s.macro(b) for b in case.block_ids])
    s.close()
    return out


CASES = {
    "cavity3d_fp64": (lambda: config.cavity(3, 33, 0.05, re=100), 30),
    "cavity3d_fp32": (lambda: config.cavity(3, 33, 0.05, re=100,
                                            precision="fp32"), 30),
    "cavity3d_fp16": (lambda: config.cavity(3, 33, 0.05, re=100,
                                            precision="fp16"), 30),
    "cavity2d_fp64": (lambda: config.cavity(2, 65, 0.05, re=100), 50),
    "lchannel": (lambda: config.lchannel(leg=14, side=9, depth=7), 20),
    "swap": (lambda: config.cavity(3, 20, 0.05, re=100,
                                   scheme="Scheme_StreamCollision_Swap"), 7),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_wide_offset_kernels_match_narrow(gpu_lib, name):
    build, steps = CASES[name]
    fa, ma = run(build(), steps, wide=False)
    fb, mb = run(build(), steps, wide=True)
    for x, y in zip(fa, fb):
        assert np.array_equal(x, y), name
    for qa, qb in zip(ma, mb):
        for x, y in zip(qa, qb):
            assert np.array_equal(x, y), name


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_block_beyond_2_31_elements(gpu_lib, precision):
    case = config.cavity(3, 1024, 0.05, re=400, wall="HalfwayBounceBack",
                         precision=precision)
    case.block_sizes = [(1024, 1024, 130)]
    s = Solver(case)
    s.init_macro(0)                # rho = 1, u = 0 everywhere
    m0 = s.mass()
    s.stream_collision(6)
    assert s.check_health() == abi.OK
    tol = 1e-10 if precision == "fp64" else 1e-6
    assert abs(s.mass() - m0) < tol * m0
    s.close()
