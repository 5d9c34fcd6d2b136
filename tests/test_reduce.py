"""FP64 reductions on the GPU (eio_reduce64) against numpy FP64 sums: dot
products (FP32 and FP64 inputs), squared differences, host arrays staged in
several chunks, device arrays, reproducibility, argument errors."""
import ctypes

import numpy as np
import pytest

from elastic_isotropic_operators_b200 import _lib, fwi

pytestmark = pytest.mark.gpu


def _call(op, x, y, on_device=False, dtype=None):
    L = _lib.lib()
    r = ctypes.c_double()
    if on_device:
        dt = 0 if x.dtype == __import__("torch").float32 else 1
        _lib.check(L.eio_reduce64(0, op, dt, x.data_ptr(), y.data_ptr(), x.numel(), 1, ctypes.byref(r)))
    else:
        dt = 0 if x.dtype == np.float32 else 1
        _lib.check(L.eio_reduce64(0, op, dt, x.ctypes.data, y.ctypes.data, x.size, 0, ctypes.byref(r)))
    return r.value


@pytest.mark.parametrize("n", [1, 1000, 12345677, 20_000_003])
def test_dot_and_misfit_fp32_host(n):
    rng = np.random.default_rng(n % 1000)
    x = rng.standard_normal(n).astype(np.float32)
    y = rng.standard_normal(n).astype(np.float32)
    want_dot = float(np.dot(x.astype(np.float64), y.astype(np.float64)))
    d = x.astype(np.float64) - y.astype(np.float64)
    want_mis = float(np.dot(d, d))
    got_dot, got_mis = _call(0, x, y), _call(1, x, y)
    scale = float(np.abs(x).astype(np.float64) @ np.abs(y).astype(np.float64))
    assert abs(got_dot - want_dot) <= 1e-10 * scale          # FP64 sums in another order
    assert abs(got_mis - want_mis) <= 1e-10 * want_mis
    assert _call(0, x, y) == got_dot   # same order every time
    assert fwi.dot64(x, y) == got_dot and fwi.misfit64(x, y) == got_mis


def test_fp64_inputs_and_norm():
    rng = np.random.default_rng(5)
    x = rng.standard_normal(3_000_001)
    got = _call(0, x, x)
    assert abs(got - float(np.dot(x, x))) <= 1e-12 * got
    assert fwi.dot64(x, x) == got


def test_device_arrays():
    import torch
    rng = np.random.default_rng(9)
    x = rng.standard_normal(5_000_000).astype(np.float32)
    y = rng.standard_normal(5_000_000).astype(np.float32)
    tx, ty = torch.from_numpy(x).cuda(), torch.from_numpy(y).cuda()
    assert _call(0, tx, ty, on_device=True) == _call(0, x, y)   # same grid, same order
    assert _call(1, tx, ty, on_device=True) == _call(1, x, y)


def test_bad_arguments():
    x = np.zeros(4, np.float32)
    L = _lib.lib()
    r = ctypes.c_double()
    assert L.eio_reduce64(0, 2, 0, x.ctypes.data, x.ctypes.data, 4, 0, ctypes.byref(r)) != 0
    assert L.eio_reduce64(0, 0, 3, x.ctypes.data, x.ctypes.data, 4, 0, ctypes.byref(r)) != 0
    assert L.eio_reduce64(0, 0, 0, None, x.ctypes.data, 4, 0, ctypes.byref(r)) != 0
    assert L.eio_reduce64(0, 0, 0, x.ctypes.data, x.ctypes.data, 0, 0, ctypes.byref(r)) == 0 and r.value == 0.0
