"""The CPU checker of the warm-start network (oracle/nn_oracle.py), pinned
without a GPU: its convolution against PyTorch's, its bf16 rounding against
PyTorch's, and its backward pass against central finite differences."""
import numpy as np
import pytest

from oracle import nn_oracle as nno


def he_params(seed):
    rng = np.random.default_rng(seed)
    w_off, b_off, total = nno.offsets()
    p = np.zeros(total)
    for l, (cin, cout, taps, relu) in enumerate(nno.LAYERS):
        sd = np.sqrt(2.0 / (taps * cin)) if relu else 0.1 / np.sqrt(taps * cin)
        p[w_off[l]:w_off[l] + cout * taps * cin] = rng.normal(
            0, sd, cout * taps * cin)
        p[b_off[l]:b_off[l] + cout] = rng.normal(0, 0.05, cout)
    return p


def test_layer_table_matches_the_network():
    assert len(nno.LAYERS) == 15
    _, _, total = nno.offsets()
    assert total == sum(co * t * ci + co for ci, co, t, _ in nno.LAYERS)


def test_conv_matches_torch():
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(1)
    x = rng.standard_normal((2, 8, 8, 5))
    w = rng.standard_normal((4, 9, 5))
    b = rng.standard_normal(4)
    y = nno.conv(x, w, b, 9)
    W = torch.from_numpy(w).reshape(4, 3, 3, 5).permute(0, 3, 1, 2)
    ref = torch.nn.functional.conv2d(torch.from_numpy(x).permute(0, 3, 1, 2),
                                     W, torch.from_numpy(b), padding=1)
    assert np.allclose(y, ref.permute(0, 2, 3, 1).numpy(), atol=1e-12)


def test_bf16_rounding_matches_torch():
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(2)
    a = np.concatenate([rng.standard_normal(10000) * 10.0 ** rng.integers(
        -20, 20, 10000), [0.0, -0.0, 1.0, 1.00390625, 1.01171875]])
    ref = torch.from_numpy(a.astype(np.float32)).to(torch.bfloat16).float()
    assert np.array_equal(nno.bf16_round(a), ref.double().numpy())


def test_backward_matches_finite_differences():
    """Directional derivative along random directions and single weights of
    three layers, on a 32 x 32 grid (the network is size-agnostic)."""
    rng = np.random.default_rng(3)
    p = he_params(4)
    cond = rng.uniform(0, 1, (2, 3))
    target = rng.standard_normal((2, 32, 32, 3)) * 0.5
    loss, _, g = nno.loss_and_grads(p, cond, target, size=32)
    eps = 1e-5
    for k in range(2):
        v = rng.standard_normal(p.size)
        v /= np.linalg.norm(v)
        lp = nno.loss_and_grads(p + eps * v, cond, target, 32,
                                need_grads=False)[0]
        lm = nno.loss_and_grads(p - eps * v, cond, target, 32,
                                need_grads=False)[0]
        fd = (lp - lm) / (2 * eps)
        assert abs(fd - g @ v) <= 1e-5 * abs(g @ v) + 1e-9, (fd, g @ v)
    w_off, b_off, _ = nno.offsets()
    for l in (0, 7, 14):
        idx = [w_off[l] + 3, b_off[l]]
        for i in idx:
            e = np.zeros(p.size)
            e[i] = 1e-7    # small enough that no ReLU changes side
            lp = nno.loss_and_grads(p + e, cond, target, 32,
                                    need_grads=False)[0]
            lm = nno.loss_and_grads(p - e, cond, target, 32,
                                    need_grads=False)[0]
            fd = (lp - lm) / 2e-7
            assert abs(fd - g[i]) <= 2e-4 * abs(g[i]) + 2e-9, (l, i, fd, g[i])
