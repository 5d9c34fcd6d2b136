"""CPU oracle of the learned preconditioner's network -- TEST INFRASTRUCTURE.

Only tests/ (and __graft_entry__.smoke()) import this module, as the checker
of the CUDA kernels in eio_cnn.cu; the product package never imports it.

The reference has no learned component, so nothing in the reference tree pins
this oracle; it is pinned instead by the identities it must satisfy (tests:
central differences of the loss against ``backward``'s weight and input
gradients in FP64, and the adjoint identity <conv(x), y> = <x, conv_T(y)>).

Conventions (those of the kernels): activations NHWC, weights [9][Cout][Cin]
with tap = 3 dy + dx, y[p][co] = sum_tap sum_ci x[p + (dy - 1, dx - 1)][ci]
w[tap][co][ci], zero padding, no bias, ReLU after every layer but the last.
"""
import numpy as np


def bf16_round(a):
    """Round FP32 values to BF16 (nearest, ties to even), returned as float32."""
    a = np.ascontiguousarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    nan = np.isnan(a)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    out = r.astype(np.uint32).view(np.float32).copy()
    out[nan] = np.nan
    return out


def conv3x3(x, w):
    """x [N][H][W][Cin], w [9][Cout][Cin] -> [N][H][W][Cout] (FP64)."""
    x = np.asarray(x, np.float64)
    w = np.asarray(w, np.float64)
    n, h, wd, _ = x.shape
    xp = np.zeros((n, h + 2, wd + 2, x.shape[3]))
    xp[:, 1:-1, 1:-1] = x
    y = np.zeros((n, h, wd, w.shape[1]))
    for tap in range(9):
        dy, dx = divmod(tap, 3)
        y += xp[:, dy:dy + h, dx:dx + wd] @ w[tap].T
    return y


def conv3x3_transpose(dy, w):
    """Adjoint of conv3x3 in x: dx[p][ci] = sum_tap sum_co dy[p - off(tap)][co] w[tap][co][ci]."""
    dy = np.asarray(dy, np.float64)
    w = np.asarray(w, np.float64)
    n, h, wd, _ = dy.shape
    dxp = np.zeros((n, h + 2, wd + 2, w.shape[2]))
    for tap in range(9):
        ty, tx = divmod(tap, 3)
        dxp[:, ty:ty + h, tx:tx + wd] += dy @ w[tap]
    return dxp[:, 1:-1, 1:-1]


def conv3x3_wgrad(x, dy):
    """dw[tap][co][ci] = sum_p dy[p][co] x[p + off(tap)][ci] (FP64)."""
    x = np.asarray(x, np.float64)
    dy = np.asarray(dy, np.float64)
    n, h, wd, cin = x.shape
    xp = np.zeros((n, h + 2, wd + 2, cin))
    xp[:, 1:-1, 1:-1] = x
    d2 = dy.reshape(-1, dy.shape[3])
    dw = np.zeros((9, dy.shape[3], cin))
    for tap in range(9):
        ty, tx = divmod(tap, 3)
        dw[tap] = d2.T @ xp[:, ty:ty + h, tx:tx + wd].reshape(-1, cin)
    return dw


def _keep(v):
    return v


def _bf16_64(v):
    return bf16_round(np.asarray(v, np.float32)).astype(np.float64)


def forward(x, ws, bf16=False):
    """Activations of every layer: a[0] = x, a[l] = relu(conv(a[l-1], w_l)) for
    l < L, a[L] = conv(a[L-1], w_L).  bf16=True rounds the hidden activations
    to BF16 as the kernels store them."""
    r = _bf16_64 if bf16 else _keep
    a = [np.asarray(x, np.float64)]
    for l, w in enumerate(ws):
        z = conv3x3(a[-1], w)
        a.append(r(np.maximum(z, 0.0)) if l < len(ws) - 1 else z)
    return a


def loss(y, t, nc):
    """0.5 sum over pixels and the first nc channels of (y - t)^2 / count."""
    d = np.asarray(y, np.float64)[..., :nc] - np.asarray(t, np.float64)
    return 0.5 * float((d * d).sum()) / d.size


def backward(a, ws, t, nc, bf16=False):
    """Weight gradients of ``loss`` and the gradient with respect to the input.
    bf16=True rounds the layer gradients to BF16 as the kernels store them."""
    r = _bf16_64 if bf16 else _keep
    y = a[-1]
    d = np.zeros_like(y)
    d[..., :nc] = (y[..., :nc] - np.asarray(t, np.float64)) / (y[..., :nc].size)
    d = r(d)
    grads = [None] * len(ws)
    for l in range(len(ws) - 1, -1, -1):
        grads[l] = conv3x3_wgrad(a[l], d)
        d = conv3x3_transpose(d, ws[l])
        if l > 0:
            d = r(d * (a[l] > 0))
    return grads, d


# ---------------------------------------------------------------- U-Net
# The four-level U-Net of precond.UNet: weights [Cout][9][Cin] per layer in
# the order below; encoder levels of two convolutions (the second one's
# output is the skip connection), 2x2 average pooling down, a bottleneck
# convolution, then per decoder level nearest 2x upsampling, concatenation
# [upsampled, skip] and one convolution; a linear head.
UNET_LAYERS = ("e1a", "e1b", "e2a", "e2b", "e3a", "e3b", "bott", "d3", "d2", "d1", "head")


def unet_channels(base=32, cin=16, cout=16):
    b = base
    return [(cin, b), (b, b), (b, 2 * b), (2 * b, 2 * b), (2 * b, 4 * b), (4 * b, 4 * b), (4 * b, 8 * b),
            (8 * b + 4 * b, 4 * b), (4 * b + 2 * b, 2 * b), (2 * b + b, b), (b, cout)]


def _conv(x, w):
    return conv3x3(x, np.transpose(np.asarray(w, np.float64), (1, 0, 2)))


def _convT(dy, w):
    return conv3x3_transpose(dy, np.transpose(np.asarray(w, np.float64), (1, 0, 2)))


def _wgrad(x, dy):
    return np.transpose(conv3x3_wgrad(x, dy), (1, 0, 2))


def pool2(x):
    return 0.25 * (x[:, 0::2, 0::2] + x[:, 1::2, 0::2] + x[:, 0::2, 1::2] + x[:, 1::2, 1::2])


def pool2_adj(dy):
    return np.repeat(np.repeat(0.25 * dy, 2, axis=1), 2, axis=2)


def up2(x):
    return np.repeat(np.repeat(x, 2, axis=1), 2, axis=2)


def up2_adj(dy):
    return dy[:, 0::2, 0::2] + dy[:, 1::2, 0::2] + dy[:, 0::2, 1::2] + dy[:, 1::2, 1::2]


def unet_forward(x, ws, bf16=False):
    """Every activation of the U-Net (a dict); 'y' is the head output.
    bf16=True rounds every stored activation to BF16 where the kernels do."""
    r = _bf16_64 if bf16 else _keep
    a = {"x": np.asarray(x, np.float64)}
    relu = lambda z: r(np.maximum(z, 0.0))
    a["e1a"] = relu(_conv(a["x"], ws[0]))
    a["s1"] = relu(_conv(a["e1a"], ws[1]))
    a["p1"] = r(pool2(a["s1"]))
    a["e2a"] = relu(_conv(a["p1"], ws[2]))
    a["s2"] = relu(_conv(a["e2a"], ws[3]))
    a["p2"] = r(pool2(a["s2"]))
    a["e3a"] = relu(_conv(a["p2"], ws[4]))
    a["s3"] = relu(_conv(a["e3a"], ws[5]))
    a["p3"] = r(pool2(a["s3"]))
    a["b"] = relu(_conv(a["p3"], ws[6]))
    a["c3"] = np.concatenate([up2(a["b"]), a["s3"]], axis=-1)
    a["d3"] = relu(_conv(a["c3"], ws[7]))
    a["c2"] = np.concatenate([up2(a["d3"]), a["s2"]], axis=-1)
    a["d2"] = relu(_conv(a["c2"], ws[8]))
    a["c1"] = np.concatenate([up2(a["d2"]), a["s1"]], axis=-1)
    a["d1"] = relu(_conv(a["c1"], ws[9]))
    a["y"] = _conv(a["d1"], ws[10])
    return a


def unet_backward(a, ws, t, nc, bf16=False):
    """Weight gradients (list, [Cout][9][Cin]) of ``loss(a['y'], t, nc)``."""
    r = _bf16_64 if bf16 else _keep
    y = a["y"]
    d = np.zeros_like(y)
    d[..., :nc] = (y[..., :nc] - np.asarray(t, np.float64)) / (y[..., :nc].size)
    d = r(d)
    g = [None] * len(ws)
    g[10] = _wgrad(a["d1"], d)
    dd1 = r(_convT(d, ws[10]))

    def layer(k, xin, yout, dy):
        dz = dy * (yout > 0)
        g[k] = _wgrad(xin, dz)
        return r(_convT(dz, ws[k]))

    dc1 = layer(9, a["c1"], a["d1"], dd1)
    cu1 = a["d2"].shape[-1]
    dd2, ds1 = r(up2_adj(dc1[..., :cu1])), dc1[..., cu1:]
    dc2 = layer(8, a["c2"], a["d2"], dd2)
    cu2 = a["d3"].shape[-1]
    dd3, ds2 = r(up2_adj(dc2[..., :cu2])), dc2[..., cu2:]
    dc3 = layer(7, a["c3"], a["d3"], dd3)
    cu3 = a["b"].shape[-1]
    db, ds3 = r(up2_adj(dc3[..., :cu3])), dc3[..., cu3:]
    dp3 = layer(6, a["p3"], a["b"], db)
    ds3 = r(ds3 + pool2_adj(dp3))
    de3a = layer(5, a["e3a"], a["s3"], ds3)
    dp2 = layer(4, a["p2"], a["e3a"], de3a)
    ds2 = r(ds2 + pool2_adj(dp2))
    de2a = layer(3, a["e2a"], a["s2"], ds2)
    dp1 = layer(2, a["p1"], a["e2a"], de2a)
    ds1 = r(ds1 + pool2_adj(dp1))
    de1a = layer(1, a["e1a"], a["s1"], ds1)
    dz = de1a * (a["e1a"] > 0)
    g[0] = _wgrad(a["x"], dz)
    return g
