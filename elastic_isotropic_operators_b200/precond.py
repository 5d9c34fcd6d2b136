"""Learned FWI preconditioner: a small convolutional network that maps an FWI
gradient to an approximate Gauss-Newton model update, trained on pairs that
the Born operators produce, with the exact misfit accepting or rejecting each
learned step (``fwi.lbfgs(..., precond=...)``).

The reference has no learned component (its FWI scripts run pySolver's
L-BFGS on the plain gradient); the network and its kernels are this
library's.  Training pairs: for a background m0 and seeded smooth
perturbations dm, the Born forward then adjoint gives g = J^T J dm, the
Gauss-Newton Hessian applied to dm; the network learns dm from g.  Near m0
the FWI gradient is g = J^T J (m - m_true) to first order, so the learned
update is -net(g).

Features per pixel (16 input channels, 4 used): the three gradient channels
relative to the background scale (g_c * mean(m0_c)), divided by their RMS
over the model, and an illumination map (the Born normal operator applied to
a constant relative perturbation, normalised to a maximum of 1).  Targets:
the relative perturbation dm_c / mean(m0_c) times K / RMS(features), K fixed
on the training set so that the targets are O(1).  Two networks, both with
BF16 weights and activations, FP32 accumulation, FP32 master weights with
Adam, no biases, 3 of 16 output channels used:
  * ConvNet: a plain stack of 3x3 convolutions 16 -> 32 -> ... -> 32 -> 16
    with ReLU between layers (``eio_cnn_*`` kernels);
  * UNet: the four-level U-Net (32 / 64 / 128 / 256 channels, pooling,
    upsampling, concatenated skips), every convolution an implicit GEMM on
    tcgen05 (``eio_unet_*`` kernels); ``LearnedPreconditioner(arch="unet")``.
Every product runs in the library's kernels; torch only holds the device
memory and the stream.
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import check

__all__ = ["ConvNet", "UNet", "unet_channels", "unet_pad_shape", "LearnedPreconditioner", "smooth_perturbation"]

_CIN = 16    # input channels of the first layer (4 features used)
_COUT = 16   # output channels of the last layer (3 used)


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise _lib.EioError(-3, "the learned preconditioner needs a CUDA device")
    return torch


def _p(t):
    return ctypes.c_void_p(int(t.data_ptr()))


class ConvNet:
    """The network: ``hidden`` channels, ``depth`` 3x3 convolutions (depth >= 2).
    Weights [9][Cout][Cin]: FP32 master copies, BF16 working copies, Adam moments."""

    def __init__(self, depth=6, hidden=32, nin=4, nout=3, device=0, seed=0):
        torch = _torch()
        if depth < 2 or hidden not in (16, 32) or not (1 <= nin <= _CIN) or not (1 <= nout <= _COUT):
            raise ValueError("depth >= 2, hidden 16 or 32, 1 <= nin <= 16, 1 <= nout <= 16")
        self.dev = torch.device("cuda", device)
        self.nin, self.nout = nin, nout
        self.chans = [_CIN] + [hidden] * (depth - 1) + [_COUT]
        rng = np.random.default_rng(seed)
        self.w32, self.wb, self.wt, self.m, self.v, self.dw = [], [], [], [], [], []
        for l in range(depth):
            ci, co = self.chans[l], self.chans[l + 1]
            fan = 9 * (nin if l == 0 else ci)
            w = rng.standard_normal((9, co, ci)) * np.sqrt(2.0 / fan)
            if l == 0:
                w[:, :, nin:] = 0.0
            if l == depth - 1:
                w *= 0.1
                w[:, nout:, :] = 0.0
            w32 = torch.tensor(w, dtype=torch.float32, device=self.dev)
            self.w32.append(w32)
            self.wb.append(w32.to(torch.bfloat16))
            self.wt.append(torch.empty((9, ci, co), dtype=torch.bfloat16, device=self.dev))
            self.m.append(torch.zeros_like(w32))
            self.v.append(torch.zeros_like(w32))
            self.dw.append(torch.zeros_like(w32))
        self.step = 0
        self._shape = None
        self._loss = torch.zeros(1, dtype=torch.float64, device=self.dev)
        self._part = torch.zeros(1024, dtype=torch.float64, device=self.dev)

    # ------------------------------------------------------------ buffers
    def _buffers(self, n, h, w):
        if self._shape == (n, h, w):
            return
        torch = _torch()
        bf = torch.bfloat16
        self.act = [None] + [torch.empty((n, h, w, c), dtype=bf, device=self.dev) for c in self.chans[1:]]
        self.y32 = torch.empty((n, h, w, _COUT), dtype=torch.float32, device=self.dev)
        self.dz = [torch.empty((n, h, w, c), dtype=bf, device=self.dev) for c in self.chans[1:]]
        need = ctypes.c_longlong()
        nmax = 0
        for l in range(len(self.chans) - 1):
            check(_lib.lib().eio_cnn_wgrad_scratch(n, h, w, self.chans[l], self.chans[l + 1], ctypes.byref(need)))
            nmax = max(nmax, need.value)
        self.scratch = torch.empty(nmax, dtype=torch.float32, device=self.dev)
        self._shape = (n, h, w)

    def _stream(self):
        return ctypes.c_void_p(_torch().cuda.current_stream(self.dev).cuda_stream)

    # ------------------------------------------------------------ passes
    def forward(self, x):
        """x: BF16 [N][H][W][16] (device) -> FP32 [N][H][W][16] (device; the
        first ``nout`` channels are the output)."""
        L = _lib.lib()
        torch = _torch()
        n, h, w, c = x.shape
        if c != _CIN or x.dtype != torch.bfloat16 or not x.is_contiguous() or x.device != self.dev:
            raise ValueError("input must be a contiguous BF16 [N][H][W][%d] tensor on %s" % (_CIN, self.dev))
        self._buffers(n, h, w)
        st = self._stream()
        self.act[0] = x
        last = len(self.chans) - 2
        for l in range(last + 1):
            check(L.eio_cnn_conv3x3(n, h, w, self.chans[l], self.chans[l + 1], _p(self.act[l]), _p(self.wb[l]),
                                    None, int(l < last), _p(self.act[l + 1]),
                                    _p(self.y32) if l == last else None, st))
        return self.y32

    def backward(self, target):
        """Weight gradients of 0.5 mean((y - target)^2) over the first nout
        channels (target FP32 [N][H][W][nout], device) after ``forward``.
        Returns the loss as a device scalar (FP64)."""
        L = _lib.lib()
        torch = _torch()
        n, h, w = self._shape
        if tuple(target.shape) != (n, h, w, self.nout) or target.dtype != torch.float32 or \
                not target.is_contiguous():
            raise ValueError("target must be a contiguous FP32 [%d][%d][%d][%d] tensor" % (n, h, w, self.nout))
        st = self._stream()
        depth = len(self.chans) - 1
        check(L.eio_cnn_mse(n * h * w, _COUT, self.nout, _p(self.y32), _p(target), _p(self.dz[-1]),
                            _p(self._part), _p(self._loss), st))
        for l in range(depth - 1, -1, -1):
            ci, co = self.chans[l], self.chans[l + 1]
            check(L.eio_cnn_conv3x3_wgrad(n, h, w, ci, co, _p(self.act[l]), _p(self.dz[l]), _p(self.dw[l]),
                                          _p(self.scratch), self.scratch.numel(), st))
            if l > 0:
                check(L.eio_cnn_flip(ci, co, _p(self.wb[l]), _p(self.wt[l]), st))
                check(L.eio_cnn_conv3x3(n, h, w, co, ci, _p(self.dz[l]), _p(self.wt[l]), _p(self.act[l]), 0,
                                        _p(self.dz[l - 1]), None, st))
        return self._loss

    def adam(self, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
        L = _lib.lib()
        st = self._stream()
        self.step += 1
        for l in range(len(self.w32)):
            check(L.eio_cnn_adam(self.w32[l].numel(), _p(self.w32[l]), _p(self.m[l]), _p(self.v[l]),
                                 _p(self.dw[l]), lr, b1, b2, eps, self.step, _p(self.wb[l]), st))

    def weights(self):
        """FP32 master weights as numpy arrays [9][Cout][Cin]."""
        return [w.cpu().numpy() for w in self.w32]

    def set_weights(self, ws):
        torch = _torch()
        for l, w in enumerate(ws):
            self.w32[l].copy_(torch.as_tensor(np.asarray(w, np.float32)))
            self.wb[l].copy_(self.w32[l].to(torch.bfloat16))


def _tma_level_ok(h, w):
    """The U-Net kernels' TMA boxes tile an h x w image: 128-pixel convolution
    tiles and 64-pixel weight-gradient slices are rectangles of it (widths that
    are multiples of the box or divide it, heights the rectangle divides)."""
    for px in (128, 64):
        if w % px and not (px % w == 0 and h % (px // w) == 0):
            return False
    return True


def unet_pad_shape(h, w, levels=4, slack=0.15):
    """(h', w') >= (h, w), multiples of 2^(levels-1): the smallest such shape
    within ``slack`` more pixels whose every level (h / 2^l, w / 2^l) the TMA
    kernels tile (e.g. 3400 x 1000 -> 3400 x 1024); else the sizes rounded up to
    the multiple (the copy-loop kernel takes those)."""
    m = 1 << (levels - 1)
    h0, w0 = -(-h // m) * m, -(-w // m) * m
    best = None
    for hh in range(h0, int(h * (1 + slack)) + 1, m):
        for ww in range(w0, int(w * (1 + slack)) + 1, m):
            if hh * ww > (1 + slack) * h * w or (best is not None and hh * ww >= best[0] * best[1]):
                continue
            if all(_tma_level_ok(hh >> l, ww >> l) for l in range(levels)):
                best = (hh, ww)
    return best if best is not None else (h0, w0)


def unet_channels(base=32):
    """(cin, cout) of the U-Net's eleven 3x3 convolutions: two per encoder level
    (base, 2 base, 4 base channels), the bottleneck (8 base), one per decoder
    level on the concatenation [upsampled, skip], and the head."""
    b = base
    return [(_CIN, b), (b, b), (b, 2 * b), (2 * b, 2 * b), (2 * b, 4 * b), (4 * b, 4 * b), (4 * b, 8 * b),
            (8 * b + 4 * b, 4 * b), (4 * b + 2 * b, 2 * b), (2 * b + b, b), (b, _COUT)]


class UNet:
    """Four-level U-Net: 3x3 convolutions with ReLU, 2x2 average pooling down,
    nearest 2x upsampling up, skip connections by concatenation; base 32 gives
    channels 32 / 64 / 128 / 256 and 1.17 M parameters.  Input BF16 NHWC
    [N][H][W][16] (the gradient's three channels and the illumination, as
    ConvNet), output FP32 [N][H][W][16] (the first ``nout`` channels used); H
    and W multiples of 8 (three poolings).

    Every convolution is an implicit GEMM on the library's tcgen05 kernel
    (eio_unet_conv3x3: the 3x3 neighbourhoods gathered by the GEMM's copy
    loop) -- forward with the weights, data gradient with the flipped weights,
    weight gradient (eio_unet_conv3x3_wgrad) with both operands read in place,
    split over the pixels (fixed summation order).  Weights [Cout][9][Cin]:
    FP32 master copies with Adam, BF16 working copies.  The same interface as
    ConvNet (forward, backward, adam, weights, set_weights)."""

    multiple = 8

    def __init__(self, base=32, nin=4, nout=3, device=0, seed=0):
        torch = _torch()
        if base % 8 or base < 8 or not (1 <= nin <= _CIN) or not (1 <= nout <= _COUT):
            raise ValueError("base a multiple of 8, 1 <= nin <= 16, 1 <= nout <= 16")
        self.dev = torch.device("cuda", device)
        self.nin, self.nout, self.base = nin, nout, base
        self.chans = unet_channels(base)
        rng = np.random.default_rng(seed)
        self.w32, self.wb, self.wf, self.m, self.v, self.dw = [], [], [], [], [], []
        last = len(self.chans) - 1
        for l, (ci, co) in enumerate(self.chans):
            fan = 9 * (nin if l == 0 else ci)
            w = rng.standard_normal((co, 9, ci)) * np.sqrt(2.0 / fan)
            if l == 0:
                w[:, :, nin:] = 0.0
            if l == last:
                w *= 0.1
                w[nout:] = 0.0
            w32 = torch.tensor(w, dtype=torch.float32, device=self.dev)
            self.w32.append(w32)
            self.wb.append(w32.to(torch.bfloat16))
            self.wf.append(torch.empty((ci, 9, co), dtype=torch.bfloat16, device=self.dev))
            self.m.append(torch.zeros_like(w32))
            self.v.append(torch.zeros_like(w32))
            self.dw.append(torch.zeros_like(w32))
        self.step = 0
        self._shape = None
        self._loss = torch.zeros(1, dtype=torch.float64, device=self.dev)
        self._part = torch.zeros(1024, dtype=torch.float64, device=self.dev)

    @staticmethod
    def pad_shape(h, w):
        """The image size the network runs an h x w image at (unet_pad_shape)."""
        return unet_pad_shape(h, w)

    def n_params(self):
        return int(sum(w.numel() for w in self.w32))

    @staticmethod
    def _lvl():
        """Resolution level (0 = full) of each convolution."""
        return [0, 0, 1, 1, 2, 2, 3, 2, 1, 0, 0]

    def _buffers(self, n, h, w):
        if self._shape == (n, h, w):
            return
        if h % 8 or w % 8:
            raise ValueError("U-Net inputs need H and W multiples of 8 (got %d x %d)" % (h, w))
        torch = _torch()
        bf = torch.bfloat16
        b = self.base
        L = [(n, h, w), (n, h // 2, w // 2), (n, h // 4, w // 4), (n, h // 8, w // 8)]
        spec = dict(e1a=(0, b), s1=(0, b), p1=(1, b), e2a=(1, 2 * b), s2=(1, 2 * b), p2=(2, 2 * b),
                    e3a=(2, 4 * b), s3=(2, 4 * b), p3=(3, 4 * b), b=(3, 8 * b), u3=(2, 8 * b), c3=(2, 12 * b),
                    d3=(2, 4 * b), u2=(1, 4 * b), c2=(1, 6 * b), d2=(1, 2 * b), u1=(0, 2 * b), c1=(0, 3 * b),
                    d1=(0, b))
        t = lambda lv, c: torch.empty(L[lv] + (c,), dtype=bf, device=self.dev)
        self.a = {k: t(lv, c) for k, (lv, c) in spec.items()}     # activations
        self.g = {k: t(lv, c) for k, (lv, c) in spec.items()}     # their gradients
        self.g["y"] = t(0, _COUT)
        self.levels = L
        self.y32 = torch.empty(L[0] + (_COUT,), dtype=torch.float32, device=self.dev)
        dzmax = max(n * (h >> lv) * (w >> lv) * co for lv, (ci, co) in zip(self._lvl(), self.chans))
        self.dz = torch.empty(dzmax, dtype=bf, device=self.dev)
        need = 1
        for lv, (ci, co) in zip(self._lvl(), self.chans):
            f = ctypes.c_longlong()
            check(_lib.lib().eio_unet_wgrad_scratch(n, h >> lv, w >> lv, ci, co, ctypes.byref(f)))
            need = max(need, f.value)
        self.scratch = torch.empty(need, dtype=torch.float32, device=self.dev)
        self._shape = (n, h, w)

    def _stream(self):
        return ctypes.c_void_p(_torch().cuda.current_stream(self.dev).cuda_stream)

    def _npix(self, lv):
        n, h, w = self.levels[lv]
        return n * h * w

    def _conv(self, k, x, lv, out16=None, out32=None, relu=1):
        n, h, w = self.levels[lv]
        ci, co = self.chans[k]
        check(_lib.lib().eio_unet_conv3x3(n, h, w, ci, co, _p(x), _p(self.wb[k]),
                                          _p(out32) if out32 is not None else None,
                                          _p(out16) if out16 is not None else None, relu, self._stream()))

    def _conv_back(self, k, x, lv, y, dy, dx):
        """Layer k: input x, output y (post-ReLU; None for the head), its
        gradient dy -> the weight gradient dw[k] and, when dx is given, the
        input's gradient."""
        L = _lib.lib()
        st = self._stream()
        n, h, w = self.levels[lv]
        ci, co = self.chans[k]
        if y is not None:
            check(L.eio_unet_relu_adj(n * h * w * co, _p(dy), _p(y), _p(self.dz), 0, st))
            dz = self.dz
        else:
            dz = dy
        check(L.eio_unet_conv3x3_wgrad(n, h, w, ci, co, _p(x), _p(dz), _p(self.dw[k]), _p(self.scratch),
                                       self.scratch.numel(), st))
        if dx is not None:
            check(L.eio_unet_flip(co, ci, _p(self.wb[k]), _p(self.wf[k]), st))
            check(L.eio_unet_conv3x3(n, h, w, co, ci, _p(dz), _p(self.wf[k]), None, _p(dx), 0, st))

    # ------------------------------------------------------------ passes
    def forward(self, x):
        """x: BF16 [N][H][W][16] (device) -> FP32 [N][H][W][16] (device)."""
        torch = _torch()
        n, h, w, c = x.shape
        if c != _CIN or x.dtype != torch.bfloat16 or not x.is_contiguous() or x.device != self.dev:
            raise ValueError("input must be a contiguous BF16 [N][H][W][%d] tensor on %s" % (_CIN, self.dev))
        self._buffers(n, h, w)
        L = _lib.lib()
        st = self._stream()
        a, b = self.a, self.base
        self.x = x

        def pool(src, lv, c, dst):
            nn, hh, ww = self.levels[lv]
            check(L.eio_unet_resample(0, nn, hh, ww, c, _p(src), _p(dst), 0, st))

        def up_cat(src, lv, cu, skip, cs, up, cat):
            # cat = [up2(src), skip] at level lv - 1
            nn, hh, ww = self.levels[lv]
            check(L.eio_unet_resample(2, nn, hh, ww, cu, _p(src), _p(up), 0, st))
            check(L.eio_unet_concat(0, self._npix(lv - 1), cu, cs, _p(up), 0, _p(skip), 0, _p(cat), st))

        self._conv(0, x, 0, out16=a["e1a"])
        self._conv(1, a["e1a"], 0, out16=a["s1"])
        pool(a["s1"], 0, b, a["p1"])
        self._conv(2, a["p1"], 1, out16=a["e2a"])
        self._conv(3, a["e2a"], 1, out16=a["s2"])
        pool(a["s2"], 1, 2 * b, a["p2"])
        self._conv(4, a["p2"], 2, out16=a["e3a"])
        self._conv(5, a["e3a"], 2, out16=a["s3"])
        pool(a["s3"], 2, 4 * b, a["p3"])
        self._conv(6, a["p3"], 3, out16=a["b"])
        up_cat(a["b"], 3, 8 * b, a["s3"], 4 * b, a["u3"], a["c3"])
        self._conv(7, a["c3"], 2, out16=a["d3"])
        up_cat(a["d3"], 2, 4 * b, a["s2"], 2 * b, a["u2"], a["c2"])
        self._conv(8, a["c2"], 1, out16=a["d2"])
        up_cat(a["d2"], 1, 2 * b, a["s1"], b, a["u1"], a["c1"])
        self._conv(9, a["c1"], 0, out16=a["d1"])
        self._conv(10, a["d1"], 0, out32=self.y32, relu=0)
        return self.y32

    def backward(self, target):
        """Weight gradients of 0.5 mean((y - target)^2) over the first nout
        channels (target FP32 [N][H][W][nout], device) after ``forward``.
        Returns the loss as a device scalar (FP64)."""
        torch = _torch()
        n, h, w = self._shape
        if tuple(target.shape) != (n, h, w, self.nout) or target.dtype != torch.float32 or \
                not target.is_contiguous():
            raise ValueError("target must be a contiguous FP32 [%d][%d][%d][%d] tensor" % (n, h, w, self.nout))
        L = _lib.lib()
        st = self._stream()
        a, g, b = self.a, self.g, self.base
        check(L.eio_cnn_mse(n * h * w, _COUT, self.nout, _p(self.y32), _p(target), _p(g["y"]), _p(self._part),
                            _p(self._loss), st))

        def split_up(cat_grad, lv, cu, cs, up_grad, skip_grad, src_grad):
            # [d up, d skip] = d cat (the skip's gradient overwritten); d src = up2^T (d up)
            check(L.eio_unet_concat(1, self._npix(lv), cu, cs, _p(up_grad), 0, _p(skip_grad), 0, _p(cat_grad), st))
            nn, hh, ww = self.levels[lv + 1]
            check(L.eio_unet_resample(3, nn, hh, ww, cu, _p(up_grad), _p(src_grad), 0, st))

        def pool_back(pooled_grad, lv, c, skip_grad):
            # the skip's gradient += pool^T (d pooled)
            nn, hh, ww = self.levels[lv]
            check(L.eio_unet_resample(1, nn, hh, ww, c, _p(pooled_grad), _p(skip_grad), 1, st))

        self._conv_back(10, a["d1"], 0, None, g["y"], g["d1"])
        self._conv_back(9, a["c1"], 0, a["d1"], g["d1"], g["c1"])
        split_up(g["c1"], 0, 2 * b, b, g["u1"], g["s1"], g["d2"])
        self._conv_back(8, a["c2"], 1, a["d2"], g["d2"], g["c2"])
        split_up(g["c2"], 1, 4 * b, 2 * b, g["u2"], g["s2"], g["d3"])
        self._conv_back(7, a["c3"], 2, a["d3"], g["d3"], g["c3"])
        split_up(g["c3"], 2, 8 * b, 4 * b, g["u3"], g["s3"], g["b"])
        self._conv_back(6, a["p3"], 3, a["b"], g["b"], g["p3"])
        pool_back(g["p3"], 2, 4 * b, g["s3"])
        self._conv_back(5, a["e3a"], 2, a["s3"], g["s3"], g["e3a"])
        self._conv_back(4, a["p2"], 2, a["e3a"], g["e3a"], g["p2"])
        pool_back(g["p2"], 1, 2 * b, g["s2"])
        self._conv_back(3, a["e2a"], 1, a["s2"], g["s2"], g["e2a"])
        self._conv_back(2, a["p1"], 1, a["e2a"], g["e2a"], g["p1"])
        pool_back(g["p1"], 0, b, g["s1"])
        self._conv_back(1, a["e1a"], 0, a["s1"], g["s1"], g["e1a"])
        self._conv_back(0, self.x, 0, a["e1a"], g["e1a"], None)
        return self._loss

    def adam(self, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
        L = _lib.lib()
        st = self._stream()
        self.step += 1
        for l in range(len(self.w32)):
            check(L.eio_cnn_adam(self.w32[l].numel(), _p(self.w32[l]), _p(self.m[l]), _p(self.v[l]),
                                 _p(self.dw[l]), lr, b1, b2, eps, self.step, _p(self.wb[l]), st))

    def weights(self):
        """FP32 master weights as numpy arrays [Cout][9][Cin]."""
        return [w.cpu().numpy() for w in self.w32]

    def set_weights(self, ws):
        torch = _torch()
        for l, w in enumerate(ws):
            self.w32[l].copy_(torch.as_tensor(np.asarray(w, np.float32)))
            self.wb[l].copy_(self.w32[l].to(torch.bfloat16))


def smooth_perturbation(shape, rng, sigma, interior=None):
    """Unit-RMS smooth random field [nx][nz] (Gaussian-filtered white noise),
    zero outside ``interior`` = (x0, x1, z0, z1) when given."""
    from .synthetic import gaussian_smooth
    f = gaussian_smooth(rng.standard_normal(shape), sigma)
    if interior is not None:
        x0, x1, z0, z1 = interior
        mask = np.zeros(shape)
        mask[x0:x1, z0:z1] = 1.0
        f = gaussian_smooth(mask, 2.0) * f
    return (f / np.sqrt(np.mean(f * f))).astype(np.float32)


class LearnedPreconditioner:
    """Learned approximate inverse of the Gauss-Newton Hessian at a background.

    born: a BornElasticShotsGpu on the FWI's acquisition; m0: the background
    (elastic parameters [3][nx][nz]) the pairs are generated at (it becomes
    born's background); interior: (x0, x1, z0, z1) cells where perturbations
    live (default: inside the absorbing pads).  ``__call__(m, g)`` returns the
    learned model update (a descent candidate) for the gradient g, for
    ``fwi.lbfgs(precond=...)``; it needs make_pairs (which fixes the target
    scale K) and train first."""

    def __init__(self, born, m0, interior=None, net=None, sigma=3.0, rel_rms=0.02, seed=0, arch="convnet"):
        self.born = born
        self.m0 = np.ascontiguousarray(m0, dtype=np.float32)
        self.scale = np.abs(self.m0.reshape(3, -1)).mean(axis=1).astype(np.float64)
        self.scale[self.scale == 0] = 1.0
        nx, nz = self.m0.shape[1:]
        if interior is None:
            fd = born.fd
            interior = (fd.xPadMinus + fd.fat, nx - fd.xPadPlus - fd.fat, fd.zPadMinus + fd.fat,
                        nz - fd.zPadPlus - fd.fat)
        self.interior = interior
        self.sigma, self.rel_rms = sigma, rel_rms
        if net is None:
            if arch not in ("convnet", "unet"):
                raise ValueError("arch is 'convnet' or 'unet'")
            net = ConvNet(seed=seed) if arch == "convnet" else UNet(seed=seed)
        self.net = net
        self.K = None
        self.born.setBackground(self.m0)
        self.illum = self._illumination()

    # ------------------------------------------------------------ Born pairs
    def _normal(self, dm):
        """J^T J dm at the background (Born forward, then adjoint)."""
        d = np.zeros(self.born.dataSpace().getNdArray().shape, np.float32)
        self.born.forward(False, np.ascontiguousarray(dm, np.float32), d)
        g = np.zeros_like(self.m0)
        self.born.adjoint(False, g, d)
        return g

    def _illumination(self):
        x0, x1, z0, z1 = self.interior
        u = np.zeros_like(self.m0)
        u[:, x0:x1, z0:z1] = (self.rel_rms * self.scale)[:, None, None]
        h = self._normal(u) * self.scale[:, None, None]
        e = np.sqrt((h.astype(np.float64) ** 2).sum(axis=0))
        return (e / max(e.max(), 1e-30)).astype(np.float32)

    def _rel_gradient(self, g):
        return np.asarray(g, np.float64) * self.scale[:, None, None]

    def features(self, g):
        """(NHWC feature image [nx][nz][16] FP32, RMS used) of a gradient [3][nx][nz]."""
        gr = self._rel_gradient(g)
        s = float(np.sqrt(np.mean(gr * gr)))
        s = s if s > 0 else 1.0
        f = np.zeros(self.m0.shape[1:] + (_CIN,), np.float32)
        f[..., :3] = np.moveaxis(gr / s, 0, -1)
        f[..., 3] = self.illum
        return f, s

    def make_pairs(self, nsamples, seed=1):
        """Features and targets of ``nsamples`` seeded perturbations: (X
        [n][nx][nz][16], T [n][nx][nz][3], feature RMS [n], dm [n][3][nx][nz])."""
        rng = np.random.default_rng(seed)
        shape = self.m0.shape[1:]
        X, S, D = [], [], []
        for _ in range(nsamples):
            rel = np.stack([smooth_perturbation(shape, rng, self.sigma, self.interior) for _ in range(3)])
            dm = (rel * (self.rel_rms * self.scale)[:, None, None]).astype(np.float32)
            f, s = self.features(self._normal(dm))
            X.append(f)
            S.append(s)
            D.append(dm)
        X, S, D = np.stack(X), np.array(S), np.stack(D)
        rel = D.astype(np.float64) / self.scale[None, :, None, None]
        if self.K is None:
            self.K = float(np.median(S / np.sqrt(np.mean(rel * rel, axis=(1, 2, 3)))))
        T = np.moveaxis(rel * (self.K / S)[:, None, None, None], 1, -1).astype(np.float32)
        return X, T, S, D

    def _pad(self, a):
        """[n][nx][nz][c] with zero rows / columns appended up to the size the
        network runs at (its size multiple; for the U-Net, a few percent more
        where that lets its TMA kernels tile every level); outputs are cut back."""
        if hasattr(self.net, "pad_shape"):
            hh, ww = self.net.pad_shape(a.shape[1], a.shape[2])
            px, pz = hh - a.shape[1], ww - a.shape[2]
        else:
            mult = getattr(self.net, "multiple", 1)
            px, pz = (-a.shape[1]) % mult, (-a.shape[2]) % mult
        return np.pad(a, ((0, 0), (0, px), (0, pz), (0, 0))) if px or pz else a

    # ------------------------------------------------------------ training
    def train(self, X, T, epochs=40, batch=8, lr=2e-3, seed=0):
        """Adam on shuffled mini-batches of (X, T) (numpy, as make_pairs gives
        them), the learning rate on a cosine schedule from lr to 0; returns the
        mean loss of each epoch."""
        if X.shape[0] < batch:
            raise ValueError("need at least one batch of %d pairs (got %d)" % (batch, X.shape[0]))
        torch = _torch()
        dev = self.net.dev
        Xd = torch.as_tensor(self._pad(X), device=dev).to(torch.bfloat16)
        Td = torch.as_tensor(np.ascontiguousarray(self._pad(T)), device=dev)
        n = X.shape[0]
        rng = np.random.default_rng(seed)
        hist = []
        for ep in range(epochs):
            order = rng.permutation(n)
            tot = torch.zeros((), dtype=torch.float64, device=dev)
            nb = 0
            for b0 in range(0, n - batch + 1, batch):
                idx = torch.as_tensor(order[b0:b0 + batch], device=dev)
                xb = Xd.index_select(0, idx).contiguous()
                tb = Td.index_select(0, idx).contiguous()
                self.net.forward(xb)
                tot += self.net.backward(tb)[0]
                self.net.adam(lr=lr * (0.5 * (1 + np.cos(np.pi * ep / epochs))))
                nb += 1
            hist.append(float(tot.item()) / max(nb, 1))
        return hist

    def predict(self, g):
        """Learned estimate of dm with J^T J dm = g ([3][nx][nz])."""
        if self.K is None:
            raise RuntimeError("make_pairs (and train) before predict: the target scale is not set")
        torch = _torch()
        f, s = self.features(g)
        nx, nz = f.shape[:2]
        x = torch.as_tensor(self._pad(f[None]), device=self.net.dev).to(torch.bfloat16).contiguous()
        y = self.net.forward(x)[0, :nx, :nz, :3].double().cpu().numpy()
        rel = np.moveaxis(y, -1, 0) * (s / self.K)
        return (rel * self.scale[:, None, None]).astype(np.float32)

    def __call__(self, m, g):
        return -self.predict(g)
