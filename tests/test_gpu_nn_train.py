"""The warm-start network on the GPU: loss, predictions and every layer's
gradients against the CPU oracle (oracle/nn_oracle.py, float64 arithmetic
with the GPU's bf16 storage emulated), training, the field resampling, and
what the trained network gains over a cold start.

Tolerances: predictions and loss to 5e-3 relative; per-layer gradients to
3e-2 relative L2 (fp32 accumulation in a different order flips a few bf16
roundings and ReLU decisions), and the whole gradient to cosine 0.9995."""
import math

import numpy as np
import pytest

from mplb_b200 import batch as bmod
from mplb_b200 import warmstart as ws
from oracle import nn_oracle as nno

pytestmark = pytest.mark.gpu


def smooth_targets(cond, size=128):
    """Synthetic smooth fields that depend on the conditioning."""
    c = (np.arange(size) + 0.5) / size
    X, Y = np.meshgrid(c, c)
    out = np.zeros((len(cond), size, size, 3), np.float32)
    for i, (a, b, n) in enumerate(cond):
        out[i, ..., 0] = 0.3 * np.cos(np.pi * (X + a)) * Y
        out[i, ..., 1] = np.sin(np.pi * Y * (1 + b)) * X * (1 - X) * 4
        out[i, ..., 2] = -np.sin(np.pi * X) * (Y - 0.5) * (1 + n)
    return out


@pytest.fixture(scope="module")
def torch_mod(gpu_lib):
    import torch
    return torch


def test_loss_and_gradients_match_oracle(gpu_lib, torch_mod):
    torch = torch_mod
    net = ws.Network(2)
    net.init(11)
    p = net.params().astype(np.float64)
    # non-zero biases so that they are exercised
    rng = np.random.default_rng(5)
    for cin, cout, taps, wo, bo in net.layers():
        p[bo:bo + cout] = rng.normal(0, 0.05, cout)
    net.set_params(p.astype(np.float32))
    p = net.params().astype(np.float64)
    cond = rng.uniform(0, 1, (2, 3)).astype(np.float32)
    target = smooth_targets(cond)
    tc = torch.from_numpy(cond).cuda()
    tt = torch.from_numpy(target).cuda()
    loss = net.loss_grad(tc, tt, want_loss=True)
    g = net.grads().astype(np.float64)
    ref_loss, ref_pred, ref_g = nno.loss_and_grads(p, cond, target,
                                                   emulate_bf16=True)
    assert abs(loss - ref_loss) <= 5e-3 * ref_loss, (loss, ref_loss)
    pred = net.forward(tc).cpu().numpy()
    assert np.linalg.norm(pred - ref_pred) <= 5e-3 * np.linalg.norm(ref_pred)
    for l, (cin, cout, taps, wo, bo) in enumerate(net.layers()):
        for lo, hi, what in ((wo, wo + cout * taps * cin, "W"),
                             (bo, bo + cout, "b")):
            a, r = g[lo:hi], ref_g[lo:hi]
            err = np.linalg.norm(a - r) / np.linalg.norm(r)
            assert err <= 3e-2, (l, what, err)
    cos = g @ ref_g / (np.linalg.norm(g) * np.linalg.norm(ref_g))
    assert cos >= 0.9995, cos


def test_training_reduces_loss(gpu_lib, torch_mod):
    torch = torch_mod
    rng = np.random.default_rng(6)
    cond = rng.uniform(0, 1, (16, 3)).astype(np.float32)
    tc = torch.from_numpy(cond).cuda()
    tt = torch.from_numpy(smooth_targets(cond)).cuda()
    net = ws.Network(8)
    net.init(3)
    hist, _ = ws.train(net, tc, tt, epochs=60, lr_max=2e-3, log_every=10)
    assert hist[-1][1] < 0.1 * hist[0][1], hist
    assert np.isfinite(net.params()).all()


def test_resampling_round_trip(gpu_lib, torch_mod):
    torch = torch_mod
    specs = [bmod.CavitySpec(128, 400.0, 0.05), bmod.CavitySpec(64, 100.0, 0.02),
             bmod.CavitySpec(256, 1000.0, 0.08)]
    rs, us = ws.scales(specs)
    fields = [[], [], []]
    # cavity-like fields: u = lid speed at the top wall and 0 on the others
    # (except at the top corners), v = 0 on every wall, rho free
    for s, r_, u_ in zip(specs, rs, us):
        c = (np.arange(s.n) + 0.5) / s.n
        X, Y = np.meshgrid(c, c)
        fields[0].append(1.0 + r_ * np.cos(np.pi * X) * np.cos(np.pi * Y))
        fields[1].append(u_ * Y * Y * (1.0 - (2.0 * X - 1.0) ** 8))
        fields[2].append(-u_ * np.sin(np.pi * Y) * np.sin(np.pi * X) * X)
    dev = [torch.from_numpy(np.concatenate([f.reshape(-1) for f in fl])).cuda()
           for fl in fields]
    net = ws.Network(1)
    grid = net.fields_to_grid(specs, *dev)
    back = net.grid_to_fields(specs, grid)
    # N = 128 maps node to node: exact up to the fp32 grid
    n0 = 128 * 128
    for k in range(3):
        a = back[k][:n0].cpu().numpy()
        b = dev[k][:n0].cpu().numpy()
        scale = rs[0] if k == 0 else us[0]
        assert np.abs(a - b).max() <= 1e-6 * scale
    # other sides: bicubic there and back.  rho and v are smooth and meet
    # their wall conditions; this u reaches 0 at the top corners where the
    # resampling assumes the lid speed along the whole top wall (a real
    # cavity's discontinuity), hence its looser bound.
    for k, tol in ((0, 1e-4), (1, 2e-2), (2, 1e-4)):
        err = ws.rel_l2_per_cavity(specs, back[k] - (1.0 if k == 0 else 0.0),
                                   dev[k] - (1.0 if k == 0 else 0.0))
        assert err.max() < tol, (k, err)


def test_warm_start_beats_cold_start(gpu_lib, torch_mod):
    """Train on the steady states of 96 small cavities (side 64, Re 100 to
    400, all stable), then start 16 held-out cavities from the network's
    prediction: they need fewer steps to the same residual than from rest
    and converge to the same field."""
    res, _ = ws.pipeline(count=112, seed=77, n_train=96, sizes=(64,),
                         re_range=(100.0, 400.0), max_steps=400_000,
                         epochs=150, batch=16, log=lambda m: None,
                         reference_check=True)
    assert res["train_converged"] == 96
    assert res["cold_converged"] == res["warm_converged"] == 16
    assert res["warm_node_steps"] < 0.8 * res["cold_node_steps"], res
    assert res["final_u_difference_median"] < 5e-3, res
    # both converged fields are as close to the tightly converged steady
    # state as each other
    assert res["warm_u_error_vs_reference_median"] <= \
        2.0 * res["cold_u_error_vs_reference_median"] + 1e-6, res
