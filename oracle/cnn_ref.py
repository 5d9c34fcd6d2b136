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
