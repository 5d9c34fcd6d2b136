"""Kernels of the learned preconditioner (eio_cnn.cu) against the CPU oracle
(oracle/cnn_ref.py), on the same BF16 inputs.

Bounds: the FP32 outputs of a convolution and the weight gradients are sums
of exact BF16 products in FP32, so they agree with the FP64 oracle to 2e-5
relative L2 (summation order only); BF16-stored outputs to 4e-3 (one BF16
rounding).  The whole network's loss and weight gradients, where every layer
stores BF16 activations and layer gradients, to 5e-3 of the oracle run on
the GPU's BF16 weights with the same BF16 storage (the rounding itself moves
the first layer's weight gradient by about 5 %)."""
import ctypes

import numpy as np
import pytest

from elastic_isotropic_operators_b200 import _lib
from oracle import cnn_ref as C

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _rel(a, b):
    a, b = np.ravel(a).astype(np.float64), np.ravel(b).astype(np.float64)
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def _p(t):
    return ctypes.c_void_p(int(t.data_ptr()))


def _bf(a):
    return torch.as_tensor(np.ascontiguousarray(a, np.float32), device="cuda").to(torch.bfloat16)


def _np(t):
    return t.float().cpu().numpy()


@pytest.fixture
def conv_path():
    """Runs a test with the given forward-convolution kernel, then restores the default."""
    L = _lib.lib()
    old = ctypes.c_int()
    _lib.check(L.eio_cnn_get_conv_path(ctypes.byref(old)))
    yield lambda p: _lib.check(L.eio_cnn_set_conv_path(p))
    _lib.check(L.eio_cnn_set_conv_path(old.value))


def _status():
    err = ctypes.c_int()
    _lib.check(_lib.lib().eio_cnn_status(1, ctypes.byref(err)))
    return err.value


@pytest.mark.parametrize("path", [0, 1])
@pytest.mark.parametrize("cin,cout", [(16, 16), (16, 32), (32, 16), (32, 32)])
@pytest.mark.parametrize("shape", [(2, 37, 45), (1, 8, 32), (3, 5, 70), (1, 3, 300)])
def test_conv_forward_relu_and_mask(cin, cout, shape, path, conv_path):
    conv_path(path)
    n, h, w = shape
    rng = np.random.default_rng(cin * 100 + cout + h)
    L = _lib.lib()
    x = C.bf16_round(rng.standard_normal((n, h, w, cin)))
    wt = C.bf16_round(rng.standard_normal((9, cout, cin)) * 0.2)
    mk = C.bf16_round(rng.standard_normal((n, h, w, cout)))
    ref = C.conv3x3(x, wt)
    xd, wd, md = _bf(x), _bf(wt), _bf(mk)
    y = torch.empty((n, h, w, cout), dtype=torch.bfloat16, device="cuda")
    y32 = torch.empty((n, h, w, cout), dtype=torch.float32, device="cuda")
    for relu in (0, 1):
        _lib.check(L.eio_cnn_conv3x3(n, h, w, cin, cout, _p(xd), _p(wd), None, relu, _p(y), _p(y32), None))
        torch.cuda.synchronize()
        r = np.maximum(ref, 0) if relu else ref
        assert _rel(_np(y32), r) < 2e-5, _rel(_np(y32), r)
        assert _rel(_np(y), r) < 4e-3
    _lib.check(L.eio_cnn_conv3x3(n, h, w, cin, cout, _p(xd), _p(wd), _p(md), 0, _p(y), _p(y32), None))
    torch.cuda.synchronize()
    r = ref * (mk > 0)
    assert _rel(_np(y32), r) < 2e-5
    assert _status() == 0


@pytest.mark.parametrize("cin,cout", [(16, 16), (16, 32), (32, 16), (32, 32)])
def test_weight_gradient_and_flip(cin, cout):
    n, h, w = 3, 29, 51
    rng = np.random.default_rng(7 + cin + cout)
    L = _lib.lib()
    x = C.bf16_round(rng.standard_normal((n, h, w, cin)))
    dy = C.bf16_round(rng.standard_normal((n, h, w, cout)))
    need = ctypes.c_longlong()
    _lib.check(L.eio_cnn_wgrad_scratch(n, h, w, cin, cout, ctypes.byref(need)))
    scratch = torch.empty(need.value, dtype=torch.float32, device="cuda")
    dw = torch.empty((9, cout, cin), dtype=torch.float32, device="cuda")
    xd, dyd = _bf(x), _bf(dy)
    _lib.check(L.eio_cnn_conv3x3_wgrad(n, h, w, cin, cout, _p(xd), _p(dyd), _p(dw), _p(scratch), need.value, None))
    torch.cuda.synchronize()
    first = dw.cpu().numpy().copy()
    assert _rel(first, C.conv3x3_wgrad(x, dy)) < 2e-5, _rel(first, C.conv3x3_wgrad(x, dy))
    _lib.check(L.eio_cnn_conv3x3_wgrad(n, h, w, cin, cout, _p(xd), _p(dyd), _p(dw), _p(scratch), need.value, None))
    torch.cuda.synchronize()
    assert np.array_equal(dw.cpu().numpy(), first)          # fixed summation order
    with pytest.raises(_lib.EioError):
        L_small = need.value - 1
        _lib.check(L.eio_cnn_conv3x3_wgrad(n, h, w, cin, cout, _p(xd), _p(dyd), _p(dw), _p(scratch), L_small, None))
    # data gradient = the forward kernel on the flipped weights
    wt = C.bf16_round(rng.standard_normal((9, cout, cin)) * 0.2)
    wd = _bf(wt)
    wf = torch.empty((9, cin, cout), dtype=torch.bfloat16, device="cuda")
    _lib.check(L.eio_cnn_flip(cin, cout, _p(wd), _p(wf), None))
    dx32 = torch.empty((n, h, w, cin), dtype=torch.float32, device="cuda")
    dx = torch.empty((n, h, w, cin), dtype=torch.bfloat16, device="cuda")
    _lib.check(L.eio_cnn_conv3x3(n, h, w, cout, cin, _p(dyd), _p(wf), None, 0, _p(dx), _p(dx32), None))
    torch.cuda.synchronize()
    assert _rel(_np(dx32), C.conv3x3_transpose(dy, wt)) < 2e-5


def test_argument_checks():
    L = _lib.lib()
    t = torch.zeros(64, dtype=torch.bfloat16, device="cuda")
    with pytest.raises(_lib.EioError):
        _lib.check(L.eio_cnn_conv3x3(1, 4, 4, 8, 16, _p(t), _p(t), None, 0, _p(t), None, None))   # 8 channels
    with pytest.raises(_lib.EioError):
        _lib.check(L.eio_cnn_conv3x3(1, 4, 4, 16, 16, None, _p(t), None, 0, _p(t), None, None))
    with pytest.raises(_lib.EioError):
        _lib.check(L.eio_cnn_adam(4, None, None, None, None, 1e-3, 0.9, 0.999, 1e-8, 1, None, None))


def test_network_loss_and_gradients_match_the_oracle():
    from elastic_isotropic_operators_b200.precond import ConvNet
    rng = np.random.default_rng(3)
    net = ConvNet(depth=4, hidden=32, nin=4, nout=3, seed=5)
    n, h, w = 2, 24, 40
    x = np.zeros((n, h, w, 16), np.float32)
    x[..., :4] = rng.standard_normal((n, h, w, 4))
    x = C.bf16_round(x)
    t = rng.standard_normal((n, h, w, 3)).astype(np.float32)
    xd = _bf(x)
    td = torch.as_tensor(t, device="cuda")
    y = net.forward(xd)
    loss = net.backward(td)
    torch.cuda.synchronize()
    ws = [_np(wb) for wb in net.wb]
    # the oracle with the kernels' BF16 storage of activations and layer gradients
    a = C.forward(x, ws, bf16=True)
    ref_loss = C.loss(a[-1], t, 3)
    grads, _ = C.backward(a, ws, t, 3, bf16=True)
    assert abs(float(loss.item()) - ref_loss) <= 1e-4 * ref_loss
    assert _rel(y.cpu().numpy()[..., :3], a[-1][..., :3]) < 1e-3
    for l, g in enumerate(grads):
        assert _rel(net.dw[l].cpu().numpy(), g) < 5e-3, (l, _rel(net.dw[l].cpu().numpy(), g))
    # and without BF16 storage, the rounding the network trains with
    a64 = C.forward(x, ws)
    grads64, _ = C.backward(a64, ws, t, 3)
    for l, g in enumerate(grads64):
        assert _rel(net.dw[l].cpu().numpy(), g) < 0.1
    # Adam: the loss of a learnable map (the first three input channels) goes down
    tl = torch.as_tensor(np.ascontiguousarray(x[..., :3]), device="cuda")
    net.forward(xd)
    first = float(net.backward(tl).item())
    for _ in range(40):
        net.adam(lr=3e-3)
        net.forward(xd)
        last = float(net.backward(tl).item())
    assert last < 0.5 * first, (first, last)
