"""Timeout path of the bounded device waits.

The TMA-pipelined step kernels (sweep, kind 1; persistent tile, kind 2) and
the tcgen05 convolution wait on mbarriers with a bounded number of polls.  The
reference has no device-side waits and ends the process on any CUDA error
(F/src/cudaErrors.cu:4-29); here a wait that runs out sets an error flag, the
CTA waits (with its own long bound) for the copies or MMAs it still has in
flight, frees what it holds and returns, and the host reports the error.

These tests set the compute-phase bound to zero polls, so every pipeline wait
gives up at once while the copies it waited for still complete normally (no
fault, no hang: the drain waits keep their full bound).  Each test checks
that the call reports the timeout and that the next call at the default
bound gives the same bits as before, i.e. the context stays usable."""
import ctypes

import numpy as np
import pytest

from elastic_isotropic_operators_b200 import _lib, prop, synthetic
from helpers import Ctx, reg_inputs

pytestmark = pytest.mark.gpu

TIMEOUT = -7


@pytest.fixture(scope="module")
def w():
    return synthetic.small()


def _limit(c):
    v = ctypes.c_longlong()
    _lib.check(c.L.eio_ctx_get_wait_limit(c.h, ctypes.byref(v)))
    return v.value


@pytest.mark.parametrize("cfg", [(1, 64, 8, 4), (2, 64, 8, 8)])
def test_step_kernel_wait_timeout_reports_and_recovers(w, cfg):
    c = Ctx(w)
    try:
        c.set_kernel(*cfg)
        r = reg_inputs(w, "f", seed=3)
        default = _limit(c)
        assert default > 0
        for adj in (0, 1):
            ref_m, ref_d = c.nl(adj, r["model"], r["data"], r["sp"], r["rp"])
            _lib.check(c.L.eio_ctx_set_wait_limit(c.h, 0))
            assert _limit(c) == 0
            with pytest.raises(prop.EioError) as ex:
                c.nl(adj, r["model"], r["data"], r["sp"], r["rp"])
            assert ex.value.code == TIMEOUT, str(ex.value)
            assert "timed out" in str(ex.value)
            _lib.check(c.L.eio_ctx_set_wait_limit(c.h, -1))
            assert _limit(c) == default
            m, d = c.nl(adj, r["model"], r["data"], r["sp"], r["rp"])
            got, want = (m, ref_m) if adj else (d, ref_d)
            for a, b in zip(got, want):
                np.testing.assert_array_equal(a, b)
        # the Born operators run the same kernels (and the fused imaging step)
        ref_dm, ref_bd = c.born(0, r["fine"], r["dm"], r["data"], r["sp"], r["rp"])
        _lib.check(c.L.eio_ctx_set_wait_limit(c.h, 0))
        with pytest.raises(prop.EioError) as ex:
            c.born(0, r["fine"], r["dm"], r["data"], r["sp"], r["rp"])
        assert ex.value.code == TIMEOUT
        _lib.check(c.L.eio_ctx_set_wait_limit(c.h, -1))
        _, bd = c.born(0, r["fine"], r["dm"], r["data"], r["sp"], r["rp"])
        for a, b in zip(bd, ref_bd):
            np.testing.assert_array_equal(a, b)
    finally:
        c.close()


def test_tcgen05_conv_wait_timeout_reports_and_recovers():
    torch = pytest.importorskip("torch")
    L = _lib.lib()
    old_path, old_limit = ctypes.c_int(), ctypes.c_longlong()
    _lib.check(L.eio_cnn_get_conv_path(ctypes.byref(old_path)))
    _lib.check(L.eio_cnn_get_wait_limit(ctypes.byref(old_limit)))
    err = ctypes.c_int()

    def p(t):
        return ctypes.c_void_p(int(t.data_ptr()))

    try:
        _lib.check(L.eio_cnn_set_conv_path(1))
        rng = np.random.default_rng(2)
        n, h, wd, cin, cout = 2, 40, 150, 32, 32
        x = torch.as_tensor(rng.standard_normal((n, h, wd, cin)).astype(np.float32), device="cuda").to(torch.bfloat16)
        wt = torch.as_tensor((rng.standard_normal((9, cout, cin)) * 0.1).astype(np.float32),
                             device="cuda").to(torch.bfloat16)
        y = torch.empty((n, h, wd, cout), dtype=torch.bfloat16, device="cuda")
        y32 = torch.empty((n, h, wd, cout), dtype=torch.float32, device="cuda")

        def conv():
            y32.fill_(float("nan"))
            _lib.check(L.eio_cnn_conv3x3(n, h, wd, cin, cout, p(x), p(wt), None, 1, p(y), p(y32), None))
            torch.cuda.synchronize()
            return y32.clone()

        _lib.check(L.eio_cnn_status(1, ctypes.byref(err)))
        ref = conv()
        _lib.check(L.eio_cnn_status(1, ctypes.byref(err)))
        assert err.value == 0 and torch.isfinite(ref).all()
        _lib.check(L.eio_cnn_set_wait_limit(0))
        bad = conv()
        _lib.check(L.eio_cnn_status(1, ctypes.byref(err)))
        assert err.value == 1                          # timed out, drained (not 2)
        assert not torch.equal(bad, ref)               # the output is incomplete
        _lib.check(L.eio_cnn_set_wait_limit(-1))
        good = conv()
        _lib.check(L.eio_cnn_status(1, ctypes.byref(err)))
        assert err.value == 0
        assert torch.equal(good, ref)
    finally:
        _lib.check(L.eio_cnn_set_wait_limit(old_limit.value))
        _lib.check(L.eio_cnn_set_conv_path(old_path.value))
