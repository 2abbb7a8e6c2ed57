"""One step in two parts (mplbgpu_step_begin: x faces and interior rows,
which read no halo layer beyond a y or z face; mplbgpu_step_finish: the
rows on y and z faces, deferred boundary nodes, halos) is one mplbgpu_step,
bit for bit, on single blocks, joined blocks with a pressure outlet, 2D
and the shifted forms; calls out of order are refused."""
import dataclasses

import numpy as np
import pytest

from mplb_b200 import Solver, abi, config

pytestmark = pytest.mark.gpu

CASES = {
    "cavity3d_40": lambda p: config.cavity(3, 40, 0.05, re=400, precision=p),
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
def test_step_in_two_parts_is_one_step(gpu_lib, name, prec):
    case = CASES[name](prec)
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


def test_x_face_import_refused_inside_a_step(gpu_lib):
    """The first part reads the x halo layers, so a face cut along x may
    not be imported between begin and finish; y and z faces may."""
    import ctypes
    import torch
    case = dataclasses.replace(config.cavity(3, 12, 0.05, re=100),
                               cuts={0: (1 << abi.SURFACES["Right"]) |
                                     (1 << abi.SURFACES["Front"])})
    case.boundaries = [b for b in case.boundaries
                       if b.surface not in ("Right", "Front")]
    s = Solver(case)
    s.init_uniform()
    lib = s.lib
    bufs = {}
    for surf in ("Right", "Front"):
        n = ctypes.c_longlong()
        eb = ctypes.c_int()
        assert lib.mplbgpu_face_size(s.h, 0, abi.SURFACES[surf],
                                     ctypes.byref(n), ctypes.byref(eb)) == 0
        bufs[surf] = torch.zeros(n.value * eb.value, dtype=torch.uint8,
                                 device="cuda")
    assert lib.mplbgpu_step_begin(s.h) == abi.OK
    assert lib.mplbgpu_import_face(s.h, 0, abi.SURFACES["Front"],
                                   bufs["Front"].data_ptr()) == abi.OK
    assert lib.mplbgpu_import_face(s.h, 0, abi.SURFACES["Right"],
                                   bufs["Right"].data_ptr()) == abi.ERR_STATE
    assert lib.mplbgpu_step_finish(s.h) == abi.OK
    s.close()
