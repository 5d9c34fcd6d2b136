"""The U-Net layer kernels (eio_gemm.cu) and the whole network (precond.UNet)
against numpy and the oracle on the same BF16 inputs.

* GEMM C = A B^T: FP32 accumulation of exact BF16 products agrees with the
  FP64 product to 1e-5 relative L2 (summation order only); ragged M, N, K,
  every tile width, split-K (slices added in a fixed order: bitwise
  reproducible), the BF16 output with ReLU and with the ReLU-derivative mask.
* The implicit-GEMM 3x3 convolution and its weight gradient: 1e-5 against
  FP64 on every channel width of the U-Net, pixel counts off the tile size.
* Weight flip, pooling / upsampling and concatenation with their adjoints:
  exact (copies, or one BF16 rounding of the same FP32 sum).
* The whole network: every layer on the network's own tensors, then end to
  end within the network's own rounding sensitivity; training lowers the
  loss."""
import ctypes

import numpy as np
import pytest

from elastic_isotropic_operators_b200 import _lib
from oracle import cnn_ref as C

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _p(t):
    return ctypes.c_void_p(int(t.data_ptr())) if t is not None else None


def _bf(a):
    return torch.as_tensor(np.ascontiguousarray(a, np.float32), device="cuda").to(torch.bfloat16)


def _np(t):
    return t.float().cpu().numpy().astype(np.float64)


def _rel(a, b):
    a, b = np.ravel(a).astype(np.float64), np.ravel(b).astype(np.float64)
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def _status_clear():
    err = ctypes.c_int()
    _lib.check(_lib.lib().eio_gemm_status(1, ctypes.byref(err)))
    return err.value


def _gemm(A, B, splits=1, c16=False, relu=0, mask=None):
    M, K = A.shape
    N = B.shape[0]
    c32 = torch.empty((M, N), dtype=torch.float32, device="cuda")
    o16 = torch.empty((M, N), dtype=torch.bfloat16, device="cuda") if c16 else None
    scratch = torch.empty((splits * M * N,), dtype=torch.float32, device="cuda") if splits > 1 else None
    _lib.check(_lib.lib().eio_gemm_bf16(M, N, K, _p(A), A.stride(0), _p(B), B.stride(0), _p(c32), _p(o16),
                                         _p(mask), relu, splits, _p(scratch), None))
    torch.cuda.synchronize()
    assert _status_clear() == 0
    return c32, o16


@pytest.mark.parametrize("M,N,K", [(128, 64, 64), (300, 100, 200), (257, 256, 1000), (64, 32, 72),
                                   (1000, 128, 576), (130, 200, 8), (5000, 16, 144), (700, 384, 256)])
def test_gemm_matches_numpy(M, N, K):
    rng = np.random.default_rng(M + N + K)
    a = C.bf16_round(rng.standard_normal((M, K)))
    b = C.bf16_round(rng.standard_normal((N, K)))
    A, B = _bf(a), _bf(b)
    want = a @ b.T
    c32, _ = _gemm(A, B)
    assert _rel(_np(c32), want) < 1e-5
    if K >= 128:
        s3, _ = _gemm(A, B, splits=3)
        assert _rel(_np(s3), want) < 1e-5
        s3b, _ = _gemm(A, B, splits=3)
        assert torch.equal(s3, s3b)                 # fixed slice order


def test_gemm_epilogues():
    rng = np.random.default_rng(4)
    M, N, K = 200, 96, 288
    a = C.bf16_round(rng.standard_normal((M, K)))
    b = C.bf16_round(rng.standard_normal((N, K)))
    A, B = _bf(a), _bf(b)
    want = a @ b.T
    c32, c16 = _gemm(A, B, c16=True, relu=1)
    assert _rel(_np(c32), np.maximum(want, 0.0)) < 1e-5
    assert np.array_equal(_np(c16), C.bf16_round(_np(c32)))
    mask = rng.standard_normal((M, N))
    c32m, _ = _gemm(A, B, mask=_bf(mask))
    assert _rel(_np(c32m), want * (C.bf16_round(mask) > 0)) < 1e-5


def test_gemm_rejects_bad_shapes():
    A = torch.zeros((64, 20), dtype=torch.bfloat16, device="cuda")
    B = torch.zeros((16, 20), dtype=torch.bfloat16, device="cuda")
    c = torch.empty((64, 16), dtype=torch.float32, device="cuda")
    with pytest.raises(_lib.EioError):
        _lib.check(_lib.lib().eio_gemm_bf16(64, 16, 20, _p(A), 20, _p(B), 20, _p(c), None, None, 0, 1, None, None))


@pytest.mark.parametrize("n,h,w,cin,cout", [(1, 5, 7, 16, 32), (2, 9, 13, 32, 16), (1, 16, 24, 96, 32),
                                             (2, 8, 8, 384, 128), (1, 4, 4, 128, 256), (3, 11, 6, 64, 64),
                                             (1, 33, 40, 16, 48), (1, 8, 16, 256, 384)])
def test_conv3x3_implicit_gemm_matches_numpy(n, h, w, cin, cout):
    """eio_unet_conv3x3 (the 3x3 taps gathered inside the GEMM): FP32 output
    against the FP64 convolution of the same BF16 values to 1e-5, the BF16
    output its rounding, ReLU; pixel counts off the 128-row tile, every
    channel width of the U-Net."""
    rng = np.random.default_rng(n * 1000 + h * 100 + cin + cout)
    x = C.bf16_round(rng.standard_normal((n, h, w, cin)))
    wt = C.bf16_round(rng.standard_normal((cout, 9, cin)) / np.sqrt(9 * cin))
    want = C._conv(x, wt)
    L = _lib.lib()
    X, W = _bf(x), _bf(wt)
    y32 = torch.empty((n, h, w, cout), dtype=torch.float32, device="cuda")
    y16 = torch.empty((n, h, w, cout), dtype=torch.bfloat16, device="cuda")
    _lib.check(L.eio_unet_conv3x3(n, h, w, cin, cout, _p(X), _p(W), _p(y32), _p(y16), 0, None))
    torch.cuda.synchronize()
    assert _rel(y32.cpu().numpy(), want) < 1e-5
    assert np.array_equal(_np(y16), C.bf16_round(y32.cpu().numpy()))
    _lib.check(L.eio_unet_conv3x3(n, h, w, cin, cout, _p(X), _p(W), _p(y32), None, 1, None))
    torch.cuda.synchronize()
    assert _rel(y32.cpu().numpy(), np.maximum(want, 0.0)) < 1e-5
    assert _status_clear() == 0


@pytest.mark.parametrize("n,h,w,cin,cout", [(1, 5, 7, 16, 32), (2, 9, 13, 32, 16), (2, 32, 32, 96, 32),
                                             (2, 8, 8, 384, 128), (1, 4, 4, 128, 256), (4, 64, 64, 32, 32),
                                             (1, 16, 16, 128, 256)])
def test_conv3x3_weight_gradient_matches_numpy(n, h, w, cin, cout):
    """eio_unet_conv3x3_wgrad (both operands read MN-major in place, the pixels
    split over the grid): against the FP64 sum to 1e-5, bitwise equal on a
    second run (fixed summation order); scratch below the split's need is
    rejected."""
    rng = np.random.default_rng(n * 7 + h + cin * 3 + cout)
    x = C.bf16_round(rng.standard_normal((n, h, w, cin)))
    dz = C.bf16_round(rng.standard_normal((n, h, w, cout)))
    want = C._wgrad(x, dz)
    L = _lib.lib()
    f = ctypes.c_longlong()
    _lib.check(L.eio_unet_wgrad_scratch(n, h, w, cin, cout, ctypes.byref(f)))
    scratch = torch.empty((max(f.value, 1),), dtype=torch.float32, device="cuda")
    dw = torch.empty((cout, 9, cin), dtype=torch.float32, device="cuda")
    X, DZ = _bf(x), _bf(dz)
    _lib.check(L.eio_unet_conv3x3_wgrad(n, h, w, cin, cout, _p(X), _p(DZ), _p(dw), _p(scratch), f.value, None))
    torch.cuda.synchronize()
    assert _rel(dw.cpu().numpy(), want) < 1e-5
    dw2 = torch.empty_like(dw)
    _lib.check(L.eio_unet_conv3x3_wgrad(n, h, w, cin, cout, _p(X), _p(DZ), _p(dw2), _p(scratch), f.value, None))
    torch.cuda.synchronize()
    assert torch.equal(dw, dw2)
    assert _status_clear() == 0
    with pytest.raises(_lib.EioError):
        _lib.check(L.eio_unet_conv3x3_wgrad(n, h, w, cin, cout, _p(X), _p(DZ), _p(dw2), _p(scratch), 0, None))


def _tma(on):
    _lib.check(_lib.lib().eio_unet_set_tma(on))


@pytest.mark.parametrize("n,h,w,cin,cout", [(2, 16, 8, 16, 32), (1, 4, 32, 32, 16), (2, 2, 64, 96, 32),
                                             (1, 3, 128, 64, 64), (1, 2, 256, 128, 256), (2, 8, 16, 384, 128),
                                             (1, 4, 32, 32, 384), (1, 8, 16, 256, 96)])
def test_conv3x3_tma_path_matches_numpy_and_the_copy_loop(n, h, w, cin, cout):
    """Shapes whose 128-pixel tiles (and 64-pixel weight-gradient slices) are
    rectangles of the image run on the TMA kernel (one 4-D box per tap and
    channel block, zero padding from the out-of-bounds fill): the convolution
    against FP64 to 1e-5 and bitwise equal to the copy-loop kernel (the same K
    order); the weight gradient against FP64 to 1e-5 and the copy loop to 1e-6
    (the pixels are split differently); the launches with up to two and four CTAs
    per SM (modes 2, 3) bitwise equal to mode 1."""
    rng = np.random.default_rng(n + 10 * h + w + cin + cout)
    x = C.bf16_round(rng.standard_normal((n, h, w, cin)))
    wt = C.bf16_round(rng.standard_normal((cout, 9, cin)) / np.sqrt(9 * cin))
    dz = C.bf16_round(rng.standard_normal((n, h, w, cout)))
    L = _lib.lib()
    X, W, DZ = _bf(x), _bf(wt), _bf(dz)
    f = ctypes.c_longlong()
    _lib.check(L.eio_unet_wgrad_scratch(n, h, w, cin, cout, ctypes.byref(f)))
    scratch = torch.empty((f.value,), dtype=torch.float32, device="cuda")
    out = {}
    mode = ctypes.c_int()
    _lib.check(L.eio_unet_get_tma(ctypes.byref(mode)))
    try:
        for on in (1, 2, 3, 0):
            _tma(on)
            y32 = torch.empty((n, h, w, cout), dtype=torch.float32, device="cuda")
            y16 = torch.empty((n, h, w, cout), dtype=torch.bfloat16, device="cuda")
            dw = torch.empty((cout, 9, cin), dtype=torch.float32, device="cuda")
            _lib.check(L.eio_unet_conv3x3(n, h, w, cin, cout, _p(X), _p(W), _p(y32), _p(y16), 1, None))
            _lib.check(L.eio_unet_conv3x3_wgrad(n, h, w, cin, cout, _p(X), _p(DZ), _p(dw), _p(scratch), f.value,
                                                None))
            torch.cuda.synchronize()
            out[on] = (y32.cpu().numpy(), _np(y16), dw.cpu().numpy())
    finally:
        _tma(mode.value)
    assert _status_clear() == 0
    want = np.maximum(C._conv(x, wt), 0.0)
    assert _rel(out[1][0], want) < 1e-5
    assert np.array_equal(out[1][0], out[0][0])
    assert np.array_equal(out[1][1], C.bf16_round(out[1][0]))
    assert _rel(out[1][2], C._wgrad(x, dz)) < 1e-5
    assert _rel(out[1][2], out[0][2]) < 1e-6
    # two or four CTAs per SM: the same tiles and splits, the same bits
    for on in (2, 3):
        assert all(np.array_equal(a, b) for a, b in zip(out[on], out[1]))


def test_flip():
    rng = np.random.default_rng(1)
    cout, cin = 24, 16
    wgt = C.bf16_round(rng.standard_normal((cout, 9, cin)))
    wf = torch.empty((cin, 9, cout), dtype=torch.bfloat16, device="cuda")
    _lib.check(_lib.lib().eio_unet_flip(cout, cin, _p(_bf(wgt)), _p(wf), None))
    torch.cuda.synchronize()
    assert np.array_equal(_np(wf), np.transpose(wgt[:, ::-1, :], (2, 1, 0)))


def test_pool_upsample_concat_and_adjoints():
    rng = np.random.default_rng(2)
    L = _lib.lib()
    n, h, w, c = 2, 6, 8, 16
    x = C.bf16_round(rng.standard_normal((n, h, w, c)))
    X = _bf(x)
    y = torch.empty((n, h // 2, w // 2, c), dtype=torch.bfloat16, device="cuda")
    _lib.check(L.eio_unet_resample(0, n, h, w, c, _p(X), _p(y), 0, None))
    want = 0.25 * (x[:, 0::2, 0::2] + x[:, 1::2, 0::2] + x[:, 0::2, 1::2] + x[:, 1::2, 1::2])
    assert np.array_equal(_np(y), C.bf16_round(want))
    yy = C.bf16_round(rng.standard_normal((n, h // 2, w // 2, c)))
    px = torch.empty_like(X)
    _lib.check(L.eio_unet_resample(1, n, h, w, c, _p(_bf(yy)), _p(px), 0, None))
    assert np.array_equal(_np(px), np.repeat(np.repeat(0.25 * yy, 2, axis=1), 2, axis=2))
    px2 = X.clone()
    _lib.check(L.eio_unet_resample(1, n, h, w, c, _p(_bf(yy)), _p(px2), 1, None))       # accumulate
    assert np.array_equal(_np(px2), C.bf16_round(x + np.repeat(np.repeat(0.25 * yy, 2, axis=1), 2, axis=2)))
    up = torch.empty((n, 2 * h, 2 * w, c), dtype=torch.bfloat16, device="cuda")
    _lib.check(L.eio_unet_resample(2, n, h, w, c, _p(X), _p(up), 0, None))
    assert np.array_equal(_np(up), np.repeat(np.repeat(x, 2, axis=1), 2, axis=2))
    du = C.bf16_round(rng.standard_normal((n, 2 * h, 2 * w, c)))
    ua = torch.empty_like(X)
    _lib.check(L.eio_unet_resample(3, n, h, w, c, _p(_bf(du)), _p(ua), 0, None))
    want = du[:, 0::2, 0::2] + du[:, 1::2, 0::2] + du[:, 0::2, 1::2] + du[:, 1::2, 1::2]
    assert np.array_equal(_np(ua), C.bf16_round(want))
    _lib.check(L.eio_unet_resample(3, n, h, w, c, _p(_bf(du)), _p(ua), 1, None))    # accumulate
    assert np.array_equal(_np(ua), C.bf16_round(C.bf16_round(want) + want))
    b = C.bf16_round(rng.standard_normal((n, h, w, 32)))
    B = _bf(b)
    z = torch.empty((n, h, w, 48), dtype=torch.bfloat16, device="cuda")
    _lib.check(L.eio_unet_concat(0, n * h * w, c, 32, _p(X), 0, _p(B), 0, _p(z), None))
    assert np.array_equal(_np(z), np.concatenate([x, b], axis=-1))
    da, db = X.clone(), torch.empty_like(B)
    _lib.check(L.eio_unet_concat(1, n * h * w, c, 32, _p(da), 1, _p(db), 0, _p(z), None))
    assert np.array_equal(_np(da), C.bf16_round(2 * x))
    assert np.array_equal(_np(db), b)
    m = C.bf16_round(rng.standard_normal((n, h, w, c)))
    r = torch.empty_like(X)
    _lib.check(L.eio_unet_relu_adj(x.size, _p(X), _p(_bf(m)), _p(r), 0, None))
    assert np.array_equal(_np(r), x * (m > 0))
    with pytest.raises(_lib.EioError):          # channels off the 16-byte chunk
        _lib.check(L.eio_unet_resample(0, n, h, w, 12, _p(X), _p(y), 0, None))
    torch.cuda.synchronize()


def _unet_case(n=2, h=32, w=64, seed=3):
    from elastic_isotropic_operators_b200 import precond
    net = precond.UNet(base=32, nin=4, nout=3, seed=seed)
    rng = np.random.default_rng(seed + 1)
    x = np.zeros((n, h, w, 16), np.float32)
    x[..., :4] = rng.standard_normal((n, h, w, 4))
    x = C.bf16_round(x)
    t = rng.standard_normal((n, h, w, 3)).astype(np.float32)
    return net, x, t


def _flips(got, want):
    """BF16 results of FP32 arithmetic against the FP64 result rounded once:
    equal but for rare one-ulp rounding flips."""
    return np.mean(got != want) < 1e-3 and _rel(got, want) < 1e-3


# (layer, input, output) of the U-Net's convolutions, by activation name
_UNET_CONVS = [(0, "x", "e1a"), (1, "e1a", "s1"), (2, "p1", "e2a"), (3, "e2a", "s2"), (4, "p2", "e3a"),
               (5, "e3a", "s3"), (6, "p3", "b"), (7, "c3", "d3"), (8, "c2", "d2"), (9, "c1", "d1"), (10, "d1", "y")]


def test_unet_layers_match_the_oracle_on_the_networks_own_tensors():
    """Every layer of a forward and backward pass checked on the GPU's own
    inputs to it (so no earlier layer's rounding carries over): convolution
    outputs, data gradients, poolings and the adjoint sums (one BF16 rounding
    of an FP32 sum against the FP64 sum rounded once: a rare one-ulp flip),
    weight gradients (FP32 against FP64 sums), upsampling + concatenation
    (exact)."""
    net, x, t = _unet_case()
    ws = [C.bf16_round(w) for w in net.weights()]
    net.forward(_bf(x))
    net.backward(torch.as_tensor(t, device="cuda"))
    torch.cuda.synchronize()
    A = {k: _np(v) for k, v in net.a.items()}
    A["x"], A["y"] = x.astype(np.float64), net.y32.cpu().numpy().astype(np.float64)
    G = {k: _np(v) for k, v in net.g.items()}
    b = net.base
    for s_, p_ in (("s1", "p1"), ("s2", "p2"), ("s3", "p3")):
        assert _flips(A[p_], C.bf16_round(C.pool2(A[s_])))
    for lo, skip, cat in (("b", "s3", "c3"), ("d3", "s2", "c2"), ("d2", "s1", "c1")):
        assert np.array_equal(A[cat], np.concatenate([C.up2(A[lo]), A[skip]], axis=-1))
    for k, xin, yout in _UNET_CONVS:
        z = C._conv(A[xin], ws[k])
        if k == 10:
            assert _rel(A["y"], z) < 1e-5, k
        else:
            assert _flips(A[yout], C.bf16_round(np.maximum(z, 0.0))), k
    # backward: the head gradient, then per layer dz = dy * (y > 0), dW and dx
    d = np.zeros_like(A["y"])
    d[..., :3] = (A["y"][..., :3] - t) / (A["y"][..., :3].size)
    assert _flips(G["y"], C.bf16_round(d))
    dy = {"y": G["y"], "d1": G["d1"], "d2": G["d2"], "d3": G["d3"], "b": G["b"], "s3": G["s3"], "e3a": G["e3a"],
          "s2": G["s2"], "e2a": G["e2a"], "s1": G["s1"], "e1a": G["e1a"]}
    for k, xin, yout in _UNET_CONVS:
        dz = dy[yout] if k == 10 else dy[yout] * (A[yout] > 0)
        assert _rel(net.dw[k].cpu().numpy(), C._wgrad(A[xin], dz)) < 1e-5, k
        if xin != "x":                         # every other input's gradient is one data-gradient GEMM
            assert _flips(G[xin], C.bf16_round(C._convT(dz, ws[k]))), k
    # the gradient's path through concatenations, upsamplings and poolings
    for cat, lo, skip, pooled, cu in (("c1", "d2", "s1", "p1", 2 * b), ("c2", "d3", "s2", "p2", 4 * b),
                                      ("c3", "b", "s3", "p3", 8 * b)):
        assert _flips(G[lo], C.bf16_round(C.up2_adj(G[cat][..., :cu])))
        assert _flips(G[skip], C.bf16_round(G[cat][..., cu:] + C.pool2_adj(G[pooled])))
    assert _status_clear() == 0


def test_unet_end_to_end_against_the_oracle():
    """Output, loss and weight gradients of the whole network against the
    oracle with BF16 rounding at the same places, and against the unrounded
    FP64 network.  The bounds are the network's own sensitivity: a 1e-7
    relative perturbation of every convolution sum (FP32-sized) moves the
    BF16 oracle's output by 2e-3 and its weight gradients by up to 1.8e-2
    (one-ulp rounding flips compound over 22 layers and ReLU masks), and BF16
    against FP64 differs by 4e-3 (output) and 6e-2 (gradients) on this case."""
    net, x, t = _unet_case()
    assert net.n_params() == sum(9 * a * b for a, b in C.unet_channels(32))
    ws = [C.bf16_round(w) for w in net.weights()]
    y = net.forward(_bf(x))
    loss = float(net.backward(torch.as_tensor(t, device="cuda")).item())
    torch.cuda.synchronize()
    got_y = y.cpu().numpy().astype(np.float64)
    got_g = [d.cpu().numpy().astype(np.float64) for d in net.dw]
    for bf16, tol_y, tol_g in ((True, 5e-3, 4e-2), (False, 1e-2, 1e-1)):
        a = C.unet_forward(x, ws, bf16=bf16)
        g = C.unet_backward(a, ws, t, 3, bf16=bf16)
        ey = _rel(got_y[..., :3], a["y"][..., :3])
        eg = [_rel(gg, w) for gg, w in zip(got_g, g)]
        print("bf16 oracle" if bf16 else "fp64 oracle", "y", ey, "grads", ["%.1e" % e for e in eg])
        assert ey < tol_y
        assert max(eg) < tol_g
        assert abs(loss - C.loss(a["y"], t, 3)) <= tol_y * C.loss(a["y"], t, 3)


def test_unet_is_deterministic_and_trains():
    """Same inputs, same bits (split-K slices in a fixed order); Adam steps on a
    fixed batch lower the loss of a learnable target (the 3x3 mean of the
    inputs: the BF16 oracle trained the same way falls from 0.060 to 0.020 in
    40 steps)."""
    net, x, _ = _unet_case(n=2, h=32, w=32, seed=5)
    xp = np.pad(x[..., :3], ((0, 0), (1, 1), (1, 1), (0, 0)))
    t = sum(xp[:, dy:dy + 32, dx:dx + 32] for dy in range(3) for dx in range(3)) / 9.0   # a learnable map
    X, T = _bf(x), torch.as_tensor(np.ascontiguousarray(t, np.float32), device="cuda")
    net.forward(X)
    net.backward(T)
    g1 = [d.clone() for d in net.dw]
    net.forward(X)
    net.backward(T)
    assert all(torch.equal(a, b) for a, b in zip(g1, net.dw))
    losses = []
    for _ in range(40):
        net.forward(X)
        losses.append(float(net.backward(T).item()))
        net.adam(lr=2e-3)
    print("loss", losses[0], losses[-1])
    assert losses[-1] < 0.6 * losses[0]


def test_unet_rejects_sizes_off_its_multiple():
    from elastic_isotropic_operators_b200 import precond
    net = precond.UNet(base=16)
    with pytest.raises(ValueError):
        net.forward(torch.zeros((1, 36, 64, 16), dtype=torch.bfloat16, device="cuda"))


def test_unet_runs_fwi_shaped_images_at_their_tma_size():
    """A 40 x 1000 image (the FWI grid's 1000-cell depth) runs at the padded
    size unet_pad_shape picks, 40 x 1024, where every level is on the TMA
    kernels: the whole network's output is bitwise that of the copy-loop
    kernel at the same size, its weight gradients within 1e-6 (the pixels are
    split differently)."""
    from elastic_isotropic_operators_b200 import precond
    h, w = precond.unet_pad_shape(40, 1000)
    assert (h, w) == (40, 1024)
    rng = np.random.default_rng(12)
    x = np.zeros((1, h, w, 16), np.float32)
    x[..., :4] = rng.standard_normal((1, h, w, 4))
    X = _bf(C.bf16_round(x))
    T = torch.as_tensor(rng.standard_normal((1, h, w, 3)).astype(np.float32), device="cuda")
    L = _lib.lib()
    mode = ctypes.c_int()
    _lib.check(L.eio_unet_get_tma(ctypes.byref(mode)))
    out = {}
    try:
        for on in (mode.value, 0):
            _tma(on)
            net = precond.UNet(seed=2)
            y = net.forward(X).clone()
            loss = float(net.backward(T).item())
            torch.cuda.synchronize()
            out[on] = (y.cpu().numpy(), loss, [d.cpu().numpy() for d in net.dw])
    finally:
        _tma(mode.value)
    assert _status_clear() == 0
    a, b = out[mode.value], out[0]
    assert np.isfinite(a[0]).all() and np.array_equal(a[0], b[0])
    assert a[1] == b[1]
    assert max(_rel(p, q) for p, q in zip(a[2], b[2])) < 1e-6
