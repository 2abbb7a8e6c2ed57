"""Tensor-core convolutions of the warm-start network (mplbnn_conv_forward,
mplbnn_conv_wgrad) against an fp64 PyTorch CPU reference of the same op on
the same bf16 inputs.

Tolerances: forward outputs are rounded to bf16 (relative half-ulp 2^-9), so
they must agree to rtol 8e-3 plus 1e-3 of the largest magnitude; weight
gradients are fp32 sums over up to 32,768 pixels, to rtol 1e-3 plus 1e-4 of
the largest magnitude."""
import ctypes

import numpy as np
import pytest

from mplb_b200 import abi

pytestmark = pytest.mark.gpu


def _torch():
    import torch
    return torch


def view(t, nimg, h, w, c, ps, coff=0):
    return abi.NNView(t.data_ptr() + coff * t.element_size(), nimg, h, w, c,
                      ps)


def ref_conv(x, wt, taps, bias, relu, mask):
    """x: (n, h, w, c) fp64, wt: (cout, taps, cin) -> (n, h, w, cout)."""
    torch = _torch()
    xt = torch.from_numpy(x).permute(0, 3, 1, 2)
    k = 3 if taps == 9 else 1
    W = torch.from_numpy(wt).reshape(wt.shape[0], k, k, wt.shape[2]).permute(
        0, 3, 1, 2)
    y = torch.nn.functional.conv2d(xt, W, padding=k // 2).permute(0, 2, 3, 1)
    y = y.numpy()
    if bias is not None:
        y = y + bias
    if relu:
        y = np.maximum(y, 0.0)
    if mask is not None:
        y = y * (mask > 0)
    return y


def ref_wgrad(dy, x, taps):
    torch = _torch()
    k = 3 if taps == 9 else 1
    xt = torch.from_numpy(x).permute(0, 3, 1, 2)
    dyt = torch.from_numpy(dy).permute(0, 3, 1, 2)
    dw = torch.nn.grad.conv2d_weight(xt, (dy.shape[3], x.shape[3], k, k), dyt,
                                     padding=k // 2)
    return dw.permute(0, 2, 3, 1).reshape(dy.shape[3], taps, x.shape[3]).numpy()


def bf16(a):
    torch = _torch()
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(
        torch.bfloat16)


def as64(t):
    return t.float().cpu().numpy().astype(np.float64)


FWD_CASES = [
    # n, h(=w), cin, cout, taps, relu, bias, in (ps, coff), out (ps, coff), f32, mask
    (2, 32, 64, 128, 9, True, True, None, None, False, False),
    (2, 64, 32, 32, 9, True, True, None, None, False, False),
    (1, 16, 256, 256, 9, True, True, None, None, False, False),
    (2, 32, 96, 192, 9, False, True, (160, 32), (200, 8), False, False),
    (1, 32, 384, 128, 9, True, False, None, None, False, True),
    (2, 128, 32, 16, 1, False, True, None, None, True, False),
    (1, 128, 16, 32, 1, False, False, None, None, False, True),
    (1, 16, 128, 384, 9, False, False, None, None, False, False),
]


@pytest.mark.parametrize("case", FWD_CASES)
def test_conv_forward_matches_reference(gpu_lib, case):
    torch = _torch()
    n, s, cin, cout, taps, relu, use_bias, inv, outv, f32, use_mask = case
    rng = np.random.default_rng(n * 100003 + s * 1009 + cin * 17 + cout)
    ips, icoff = inv or (cin, 0)
    ops, ocoff = outv or (cout, 0)
    xbuf = bf16(rng.standard_normal((n, s, s, ips))).cuda()
    wt = bf16(rng.standard_normal((cout, taps, cin)) / np.sqrt(taps * cin))
    wdev = wt.cuda()
    bias = (rng.standard_normal(cout) * 0.1).astype(np.float32)
    bdev = torch.from_numpy(bias).cuda() if use_bias else None
    dt = torch.float32 if f32 else torch.bfloat16
    ybuf = torch.zeros((n, s, s, ops), dtype=dt, device="cuda")
    mask = None
    mview = None
    if use_mask:
        mask = bf16(rng.standard_normal((n, s, s, cout))).cuda()
        mview = view(mask, n, s, s, cout, cout)
    torch.cuda.synchronize()
    rc = gpu_lib.mplbnn_conv_forward(
        ctypes.byref(view(xbuf, n, s, s, cin, ips, icoff)), wdev.data_ptr(),
        taps, bdev.data_ptr() if bdev is not None else None, int(relu),
        ctypes.byref(view(ybuf, n, s, s, cout, ops, ocoff)), int(f32),
        ctypes.byref(mview) if mview is not None else None, None)
    assert rc == 0, gpu_lib.mplbnn_error().decode()
    x = as64(xbuf)[..., icoff:icoff + cin]
    ref = ref_conv(x, as64(wt), taps, bias.astype(np.float64) if use_bias
                   else None, relu, as64(mask) if use_mask else None)
    y = as64(ybuf)
    got = y[..., ocoff:ocoff + cout]
    scale = np.abs(ref).max()
    assert np.allclose(got, ref, rtol=8e-3, atol=1e-3 * scale), (
        np.abs(got - ref).max(), scale)
    # channels outside the output view are untouched
    if outv is not None:
        assert not y[..., :ocoff].any() and not y[..., ocoff + cout:].any()


WGRAD_CASES = [
    # n, h, cout (dy), cin (x), taps, x (ps, coff)
    (2, 64, 32, 32, 9, None),
    (4, 16, 256, 128, 9, None),
    (2, 32, 128, 384, 9, None),
    (1, 128, 16, 32, 1, None),
    (2, 32, 64, 96, 9, (192, 96)),
    # few output channels: taps x input channels along M
    (2, 128, 32, 96, 9, (96, 0)),
    (3, 64, 64, 32, 9, (64, 32)),
    (1, 32, 48, 160, 9, None),
]


@pytest.mark.parametrize("case", WGRAD_CASES)
def test_conv_wgrad_matches_reference(gpu_lib, case):
    torch = _torch()
    n, s, cout, cin, taps, xv = case
    rng = np.random.default_rng(7 + n * 1009 + s * 17 + cin + cout)
    xps, xcoff = xv or (cin, 0)
    xbuf = bf16(rng.standard_normal((n, s, s, xps))).cuda()
    dy = bf16(rng.standard_normal((n, s, s, cout))).cuda()
    dw = torch.zeros((cout, taps, cin), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    rc = gpu_lib.mplbnn_conv_wgrad(
        ctypes.byref(view(dy, n, s, s, cout, cout)),
        ctypes.byref(view(xbuf, n, s, s, cin, xps, xcoff)), taps,
        dw.data_ptr(), None)
    assert rc == 0, gpu_lib.mplbnn_error().decode()
    ref = ref_wgrad(as64(dy), as64(xbuf)[..., xcoff:xcoff + cin], taps)
    got = dw.cpu().numpy().astype(np.float64)
    scale = np.abs(ref).max()
    assert np.allclose(got, ref, rtol=1e-3, atol=1e-4 * scale), (
        np.abs(got - ref).max(), scale)


def test_conv_rejects_unsupported_shapes(gpu_lib):
    torch = _torch()
    x = torch.zeros((1, 24, 24, 32), dtype=torch.bfloat16, device="cuda")
    w = torch.zeros((32, 9, 32), dtype=torch.bfloat16, device="cuda")
    y = torch.zeros_like(x)
    rc = gpu_lib.mplbnn_conv_forward(
        ctypes.byref(view(x, 1, 24, 24, 32, 32)), w.data_ptr(), 9, None, 0,
        ctypes.byref(view(y, 1, 24, 24, 32, 32)), 0, None, None)
    assert rc == abi.ERR_INVALID
    assert b"unsupported" in gpu_lib.mplbnn_error()
