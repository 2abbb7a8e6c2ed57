"""The allocation-free residual entry point, through the C ABI.

mplbgpu_residual_sums_noalloc serves callers that cannot call cudaMalloc
where they need the reduction (all device memory handed to their own pool,
or no device-wide synchronisation allowed): it takes caller-owned device
buffers and keeps its partial sums in a fixed array inside the library.
Checked against mplbgpu_residual on the same moments, on two calls in a
row (the second one also checks that q_old was replaced by q).  This file
sorts last so that a run stopping at its first failure has run every other
test before it."""
import ctypes

import numpy as np
import pytest
import torch

from mplb_b200 import Solver, abi, config

pytestmark = pytest.mark.gpu


def _noalloc(lib, q, qold):
    nv = len(q)
    qp = (ctypes.c_void_p * nv)(*[t.data_ptr() for t in q])
    op = (ctypes.c_void_p * nv)(*[t.data_ptr() for t in qold])
    sums = torch.zeros(2 * nv, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    rc = lib.mplbgpu_residual_sums_noalloc(qp, op, nv, q[0].numel(),
                                           sums.data_ptr(), stream)
    assert rc == abi.OK
    torch.cuda.synchronize()
    s = sums.cpu().numpy()
    return s[0::2] / s[1::2]


@pytest.mark.parametrize("dim,n", [(3, 40), (2, 300)])
def test_noalloc_residual_matches_residual(gpu_lib, dim, n):
    # 3D: four variables; 2D: three (rho, u, v) over 90,000 nodes, a
    # partial last CTA
    case = config.cavity(dim, n, 0.05, re=100)
    s = Solver(case)
    s.init_uniform()
    shp = s._shape(0)
    qold = [torch.ones(shp, dtype=torch.float64, device="cuda")] + [
        torch.zeros(shp, dtype=torch.float64, device="cuda")
        for _ in range(dim)]
    for _ in range(2):
        s.stream_collision(25)
        s.update_macro_vars()
        q = [torch.from_numpy(a).cuda() for a in s.macro(0)]
        _, per_ctx = s.calc_residual_error(25)
        per_na = _noalloc(gpu_lib, q, qold)
        np.testing.assert_allclose(per_na, per_ctx, rtol=1e-12, atol=0)
        for a, b in zip(qold, q):
            assert torch.equal(a, b)
    s.close()


def test_noalloc_rejects_oversize(gpu_lib):
    q = [torch.zeros(8, dtype=torch.float64, device="cuda")]
    qp = (ctypes.c_void_p * 1)(q[0].data_ptr())
    sums = torch.zeros(2, dtype=torch.float64, device="cuda")
    rc = gpu_lib.mplbgpu_residual_sums_noalloc(
        qp, qp, 1, abi.NOALLOC_MAX_NODES + 1, sums.data_ptr(), None)
    assert rc == abi.ERR_INVALID
    rc = gpu_lib.mplbgpu_residual_sums_noalloc(qp, qp, 5, 8, sums.data_ptr(),
                                               None)
    assert rc == abi.ERR_INVALID
