"""The CPU oracle of the learned preconditioner's network (oracle/cnn_ref.py),
pinned by identities: the transpose convolution is the adjoint of the
convolution, and the weight and input gradients of the loss match central
differences in FP64.  BF16 rounding matches the bit pattern rule."""
import numpy as np

from oracle import cnn_ref as C


def test_transpose_is_the_adjoint():
    rng = np.random.default_rng(0)
    x = rng.standard_normal((2, 7, 9, 5))
    y = rng.standard_normal((2, 7, 9, 4))
    w = rng.standard_normal((9, 4, 5))
    lhs = float((C.conv3x3(x, w) * y).sum())
    rhs = float((x * C.conv3x3_transpose(y, w)).sum())
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)


def test_gradients_match_central_differences():
    rng = np.random.default_rng(1)
    x = rng.standard_normal((2, 6, 5, 3))
    ws = [rng.standard_normal((9, 4, 3)) * 0.4, rng.standard_normal((9, 4, 4)) * 0.4,
          rng.standard_normal((9, 3, 4)) * 0.4]
    t = rng.standard_normal((2, 6, 5, 2))
    nc = 2
    a = C.forward(x, ws)
    grads, dx = C.backward(a, ws, t, nc)
    h = 1e-6
    for l, (w, gw) in enumerate(zip(ws, grads)):
        for idx in [(0, 0, 0), (4, 1, 2), (8, w.shape[1] - 1, w.shape[2] - 1), (3, 2, 1)]:
            wp = [v.copy() for v in ws]
            wm = [v.copy() for v in ws]
            wp[l][idx] += h
            wm[l][idx] -= h
            fd = (C.loss(C.forward(x, wp)[-1], t, nc) - C.loss(C.forward(x, wm)[-1], t, nc)) / (2 * h)
            assert abs(fd - gw[idx]) <= 1e-6 * max(abs(fd), 1e-8), (l, idx, fd, gw[idx])
    for idx in [(0, 0, 0, 0), (1, 3, 2, 1), (1, 5, 4, 2)]:
        xp, xm = x.copy(), x.copy()
        xp[idx] += h
        xm[idx] -= h
        fd = (C.loss(C.forward(xp, ws)[-1], t, nc) - C.loss(C.forward(xm, ws)[-1], t, nc)) / (2 * h)
        assert abs(fd - dx[idx]) <= 1e-6 * max(abs(fd), 1e-8)


def test_bf16_rounding():
    v = np.array([1.0, 1.00390625, 1.005859375, 1.0078125, -3.14159, 0.0, 1e-40], np.float32)
    r = C.bf16_round(v)
    assert r[0] == 1.0
    assert r[1] == 1.0                 # halfway between 1 and 1 + 2^-7: ties to even
    assert r[2] == 1.0078125           # above halfway rounds up
    assert r[3] == 1.0078125
    assert abs(r[4] + 3.140625) < 1e-7
    assert r[5] == 0.0
    assert (r.view(np.uint32) & 0xFFFF == 0).all()


def test_unet_backward_matches_central_differences():
    """The U-Net oracle (three poolings, three upsamplings, concatenated skips)
    is pinned by FP64 central differences of its loss: weight gradients of an
    encoder, the bottleneck side, a decoder and the head layer."""
    rng = np.random.default_rng(0)
    ch = C.unet_channels(8)
    ws = [rng.standard_normal((co, 9, ci)) * np.sqrt(2.0 / (9 * ci)) for ci, co in ch]
    x = rng.standard_normal((1, 8, 8, 16))
    t = rng.standard_normal((1, 8, 8, 3))
    g = C.unet_backward(C.unet_forward(x, ws), ws, t, 3)
    assert [w.shape for w in g] == [w.shape for w in ws]
    h = 1e-6
    for k, idx in ((0, (1, 4, 2)), (3, (5, 8, 7)), (4, (1, 4, 2)), (6, (60, 0, 30)), (7, (1, 4, 2)),
                   (9, (0, 3, 17)), (10, (1, 4, 2))):
        wp = [w.copy() for w in ws]
        wm = [w.copy() for w in ws]
        wp[k][idx] += h
        wm[k][idx] -= h
        fd = (C.loss(C.unet_forward(x, wp)["y"], t, 3) - C.loss(C.unet_forward(x, wm)["y"], t, 3)) / (2 * h)
        assert abs(fd - g[k][idx]) <= 1e-6 * max(abs(fd), 1e-7), (k, idx, fd, g[k][idx])


def test_unet_resampling_adjoints():
    rng = np.random.default_rng(1)
    x = rng.standard_normal((2, 6, 4, 3))
    y = rng.standard_normal((2, 3, 2, 3))
    assert np.isclose((C.pool2(x) * y).sum(), (x * C.pool2_adj(y)).sum())
    u = rng.standard_normal((2, 12, 8, 3))
    assert np.isclose((C.up2(x) * u).sum(), (x * C.up2_adj(u)).sum())
