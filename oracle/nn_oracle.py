"""CPU restatement of the warm-start network (TEST INFRASTRUCTURE ONLY).

An autograd-free numpy float64 forward and backward pass of the network in
mplb_b200/csrc/nn/warmstart.cu, on the same NHWC layouts and the same flat
parameter vector (per layer W[cout][taps][cin] then b[cout]).  It is the
checker of the tensor-core training kernels: tests compare the GPU loss and
gradients with `loss_and_grads` (optionally emulating the GPU's bf16 storage
of weights, activations and activation gradients), and `loss_and_grads` itself
is checked against central finite differences.  Only tests/ use this module.

The network has no counterpart in the reference (which has no learned
component); the oracle restates this repository's own specification:
levels of side S >> l with 32 << l channels, two 3x3 ReLU convolutions per
level, 2x2 average pooling, nearest 2x upsampling concatenated in front of
the skip connection, a 1x1 output convolution to 16 channels of which 3 are
used, mean squared error over those 3.
"""
import numpy as np

# (cin, cout, taps, relu): e0a e0 e1a e1 e2a e2 ba bb d2a d2 d1a d1 d0a d0 out
LAYERS = [(32, 32, 9, 1), (32, 32, 9, 1), (32, 64, 9, 1), (64, 64, 9, 1),
          (64, 128, 9, 1), (128, 128, 9, 1), (128, 256, 9, 1),
          (256, 256, 9, 1), (384, 128, 9, 1), (128, 128, 9, 1),
          (192, 64, 9, 1), (64, 64, 9, 1), (96, 32, 9, 1), (32, 32, 9, 1),
          (32, 16, 1, 0)]


def offsets():
    w_off, b_off, o = [], [], 0
    for cin, cout, taps, _ in LAYERS:
        w_off.append(o)
        o += cout * taps * cin
        b_off.append(o)
        o += cout
    return w_off, b_off, o


def bf16_round(a):
    """Round to the nearest bfloat16 (ties to even), returned as float64."""
    f = np.ascontiguousarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def _cols(x, taps):
    """im2col: (n, h, w, c) -> (n, h, w, taps, c); tap t = 3 kh + kw reads
    x[y + kh - 1, x + kw - 1] (zero outside)."""
    if taps == 1:
        return x[:, :, :, None, :]
    n, h, w, c = x.shape
    xp = np.zeros((n, h + 2, w + 2, c))
    xp[:, 1:-1, 1:-1] = x
    return np.stack([xp[:, t // 3:t // 3 + h, t % 3:t % 3 + w]
                     for t in range(9)], axis=3)


def _col2im(dcols, taps):
    if taps == 1:
        return dcols[:, :, :, 0, :]
    n, h, w, _, c = dcols.shape
    dxp = np.zeros((n, h + 2, w + 2, c))
    for t in range(9):
        dxp[:, t // 3:t // 3 + h, t % 3:t % 3 + w] += dcols[:, :, :, t]
    return dxp[:, 1:-1, 1:-1]


def conv(x, w, b, taps):
    cols = _cols(x, taps)
    n, h, wd = x.shape[:3]
    y = cols.reshape(n * h * wd, -1) @ w.reshape(w.shape[0], -1).T
    return y.reshape(n, h, wd, -1) + b


def conv_backward(x, w, dz, taps, need_dx=True):
    """dz: gradient at the pre-activation output -> (dx, dw, db)."""
    cols = _cols(x, taps)
    n, h, wd = x.shape[:3]
    dz2 = dz.reshape(n * h * wd, -1)
    dw = (dz2.T @ cols.reshape(n * h * wd, -1)).reshape(w.shape)
    db = dz2.sum(axis=0)
    dx = None
    if need_dx:
        dcols = (dz2 @ w.reshape(w.shape[0], -1)).reshape(cols.shape)
        dx = _col2im(dcols, taps)
    return dx, dw, db


def pool(x):
    n, h, w, c = x.shape
    return x.reshape(n, h // 2, 2, w // 2, 2, c).mean(axis=(2, 4))


def pool_backward(d):
    return np.repeat(np.repeat(d, 2, axis=1), 2, axis=2) * 0.25


def up(x):
    return np.repeat(np.repeat(x, 2, axis=1), 2, axis=2)


def up_backward(d):
    n, h, w, c = d.shape
    return d.reshape(n, h // 2, 2, w // 2, 2, c).sum(axis=(2, 4))


def inputs(cond, size=128):
    """Input planes: cond (3), x, y at node centres, zeros to 32 channels."""
    cond = np.asarray(cond, np.float64)
    n = cond.shape[0]
    x = np.zeros((n, size, size, 32))
    x[..., :3] = cond[:, None, None, :]
    c = (np.arange(size) + 0.5) / size
    x[..., 3] = c[None, None, :]
    x[..., 4] = c[None, :, None]
    return x


def unpack(params):
    w_off, b_off, _ = offsets()
    ws, bs = [], []
    for l, (cin, cout, taps, _) in enumerate(LAYERS):
        ws.append(np.asarray(params[w_off[l]:w_off[l] + cout * taps * cin],
                             np.float64).reshape(cout, taps, cin))
        bs.append(np.asarray(params[b_off[l]:b_off[l] + cout], np.float64))
    return ws, bs


def loss_and_grads(params, cond, target, size=128, emulate_bf16=False,
                   need_grads=True):
    """Mean squared error of the network on (cond, target) and its gradient
    with respect to the flat parameter vector.  target: (n, size, size, 3).
    emulate_bf16 rounds what the GPU stores in bf16 (inputs, weights,
    activations, activation gradients) and keeps float64 arithmetic."""
    r = bf16_round if emulate_bf16 else (lambda a: a)
    ws, bs = unpack(params)
    wr = [r(w) for w in ws]
    relu = lambda a: np.maximum(a, 0.0)
    act = {}

    def fwd(l, x):
        y = conv(x, wr[l], bs[l], LAYERS[l][2])
        return r(relu(y)) if LAYERS[l][3] else y

    xin = r(inputs(cond, size))
    e0a = fwd(0, xin)
    e0 = fwd(1, e0a)
    p0 = r(pool(e0))
    e1a = fwd(2, p0)
    e1 = fwd(3, e1a)
    p1 = r(pool(e1))
    e2a = fwd(4, p1)
    e2 = fwd(5, e2a)
    p2 = r(pool(e2))
    ba = fwd(6, p2)
    bb = fwd(7, ba)
    cat2 = np.concatenate([up(bb), e2], axis=3)
    d2a = fwd(8, cat2)
    d2 = fwd(9, d2a)
    cat1 = np.concatenate([up(d2), e1], axis=3)
    d1a = fwd(10, cat1)
    d1 = fwd(11, d1a)
    cat0 = np.concatenate([up(d1), e0], axis=3)
    d0a = fwd(12, cat0)
    d0 = fwd(13, d0a)
    pred = conv(d0, wr[14], bs[14], 1)
    if emulate_bf16:
        pred = pred.astype(np.float32).astype(np.float64)
    diff = pred[..., :3] - np.asarray(target, np.float64)
    count = diff.size
    loss = float((diff ** 2).sum() / count)
    if not need_grads:
        return loss, pred[..., :3], None

    w_off, b_off, total = offsets()
    grads = np.zeros(total)

    def put(l, dw, db):
        cin, cout, taps, _ = LAYERS[l]
        grads[w_off[l]:w_off[l] + cout * taps * cin] = dw.reshape(-1)
        grads[b_off[l]:b_off[l] + cout] = db

    def back(l, x, dz, mask=None, need_dx=True):
        """dz: gradient at layer l's output (pre-activation for l's own
        ReLU already folded in); returns the gradient at its input, times
        (mask > 0) when given."""
        dx, dw, db = conv_backward(x, ws[l] if not emulate_bf16 else wr[l],
                                   dz, LAYERS[l][2], need_dx)
        put(l, dw, db)
        if dx is None:
            return None
        if mask is not None:
            dx = dx * (mask > 0)
        return r(dx)

    dpred = np.zeros_like(pred)
    dpred[..., :3] = 2.0 * diff / count
    dpred = r(dpred)
    g_d0 = back(14, d0, dpred, d0)
    g_d0a = back(13, d0a, g_d0, d0a)
    g_cat0 = back(12, cat0, g_d0a)
    g_d1 = r(up_backward(g_cat0[..., :64]) * (d1 > 0))
    g_d1a = back(11, d1a, g_d1, d1a)
    g_cat1 = back(10, cat1, g_d1a)
    g_d2 = r(up_backward(g_cat1[..., :128]) * (d2 > 0))
    g_d2a = back(9, d2a, g_d2, d2a)
    g_cat2 = back(8, cat2, g_d2a)
    g_bb = r(up_backward(g_cat2[..., :256]) * (bb > 0))
    g_ba = back(7, ba, g_bb, ba)
    g_p2 = back(6, p2, g_ba)
    g_e2 = r((g_cat2[..., 256:] + pool_backward(g_p2)) * (e2 > 0))
    g_e2a = back(5, e2a, g_e2, e2a)
    g_p1 = back(4, p1, g_e2a)
    g_e1 = r((g_cat1[..., 128:] + pool_backward(g_p1)) * (e1 > 0))
    g_e1a = back(3, e1a, g_e1, e1a)
    g_p0 = back(2, p0, g_e1a)
    g_e0 = r((g_cat0[..., 64:] + pool_backward(g_p0)) * (e0 > 0))
    g_e0a = back(1, e0a, g_e0, e0a)
    back(0, xin, g_e0a, need_dx=False)
    del act
    return loss, pred[..., :3], grads
