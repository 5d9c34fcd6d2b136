"""Failure handling without a GPU fault: out of memory (a device-memory cap
makes the allocation fail on purpose), the source history in host memory
when it does not fit on the device, and NaN / Inf detection.

* Device-only history over the cap: the Born call fails with EIO_ERR_NOMEM and
  the context stays usable (the same call after lifting the cap is correct).
* Default policy over the cap: the history goes to mapped pinned host memory
  and the results are bitwise those of the device history (the kernels read
  the same values through another address); forcing host memory likewise.
* With eio_ctx_set_check_finite: a NaN in an input is rejected before any work
  (EIO_ERR_ARG); an output holding Inf after the call comes back as
  EIO_ERR_NONFINITE; without the check the same call succeeds and returns the
  Inf values."""
import ctypes

import numpy as np
import pytest

from elastic_isotropic_operators_b200 import _lib, prop, synthetic

pytestmark = pytest.mark.gpu


def _born(w, lanes=1):
    src, rec = w.geometry()
    op = prop.BornElasticShotsGpu(w.elastic, w.par, [w.source_signal()], *src, *rec)
    op.setLanes(lanes)
    return op


def _used():
    u = ctypes.c_longlong()
    _lib.check(_lib.lib().eio_get_device_memory_used(ctypes.byref(u)))
    return u.value


def _where(op):
    v = ctypes.c_int()
    _lib.check(op._L.eio_ctx_get_history_location(op.ctx, ctypes.byref(v)))
    return v.value


def _forward(op, w):
    dm = op.modelSpace()
    dm.getNdArray()[...] = w.extra["dmodel"]
    d = op.dataSpace()
    op.forward(False, dm, d)
    return d.getNdArray().copy()


def test_out_of_memory_and_the_host_history_fallback():
    w = synthetic.small(nts=120, nshots=2)
    n = w.nz * w.nx
    hist = 2 * w.nts * n * 4                    # FP32 coarse Vx / Vz history of one shot
    L = _lib.lib()
    try:
        # reference run: everything on the device; how much the call itself allocates
        ref = _born(w)
        u0 = _used()
        want = _forward(ref, w)
        assert _where(ref) == 1
        call_bytes = _used() - u0
        assert call_bytes >= hist
        # a context whose call finds room for everything but the history
        op = _born(w)
        u1 = _used()
        _lib.check(L.eio_set_device_memory_cap(u1 + (call_bytes - hist) + hist // 2))
        _lib.check(op._L.eio_ctx_set_history_location(op.ctx, 1))      # device only
        with pytest.raises(_lib.EioError) as e:
            _forward(op, w)
        assert e.value.code == -6
        # the default policy: the history moves to mapped host memory, same bits
        _lib.check(op._L.eio_ctx_set_history_location(op.ctx, 0))
        got = _forward(op, w)
        assert _where(op) == 2
        assert np.array_equal(got, want)
        # the cap lifted, device only again: the context is intact and correct
        _lib.check(L.eio_set_device_memory_cap(0))
        _lib.check(op._L.eio_ctx_set_history_location(op.ctx, 1))
        assert np.array_equal(_forward(op, w), want)
        assert _where(op) == 1
        # forced host memory, and the adjoint through it
        _lib.check(op._L.eio_ctx_set_history_location(op.ctx, 2))
        assert np.array_equal(_forward(op, w), want)
        assert _where(op) == 2
        rng = np.random.default_rng(1)
        d = op.dataSpace()
        d.getNdArray()[...] = rng.standard_normal(d.getNdArray().shape).astype(np.float32)
        g_host, g_dev = op.modelSpace(), ref.modelSpace()
        op.adjoint(False, g_host, d)
        ref.adjoint(False, g_dev, d)
        assert np.array_equal(g_host.getNdArray(), g_dev.getNdArray())
    finally:
        L.eio_set_device_memory_cap(0)


def test_the_first_call_over_the_cap_fails_and_the_context_works_after():
    """Contexts allocate at their first propagation: over the cap that call
    fails with EIO_ERR_NOMEM (whatever the history policy: the wavefields do
    not fit either) and, the cap lifted, the same context is correct."""
    w = synthetic.small(nts=60, nshots=1)
    L = _lib.lib()
    ref = _born(w)
    want = _forward(ref, w)
    op = _born(w)
    try:
        _lib.check(L.eio_set_device_memory_cap(_used() + 1024))
        with pytest.raises(_lib.EioError) as e:
            _forward(op, w)
        assert e.value.code == -6
    finally:
        L.eio_set_device_memory_cap(0)
    assert np.array_equal(_forward(op, w), want)


def test_non_finite_inputs_and_outputs():
    w = synthetic.small(nts=120, nshots=2)
    op = _born(w)
    _lib.check(op._L.eio_ctx_set_check_finite(op.ctx, 1))
    want = _forward(op, w)                      # finite in, finite out: unaffected
    dm = op.modelSpace()
    dm.getNdArray()[...] = w.extra["dmodel"]
    dm.getNdArray()[1, 30, 40] = np.nan
    d = op.dataSpace()
    with pytest.raises(_lib.EioError) as e:
        op.forward(False, dm, d)
    assert e.value.code == -1
    dd = op.dataSpace()
    dd.getNdArray()[...] = 1.0
    dd.getNdArray().reshape(-1)[7] = np.inf
    with pytest.raises(_lib.EioError) as e:
        op.adjoint(False, op.modelSpace(), dd)
    assert e.value.code == -1
    assert np.array_equal(_forward(op, w), want)   # still usable
    # the output scan: finite inputs, an output that holds Inf after the call (carried in by add = True, which
    # the input scan does not look at; a stable propagation of finite inputs cannot overflow: the injection
    # scaling keeps even a 1e38 source at about 1e25 in the data)
    src, rec = w.geometry()
    nl = prop.nonlinearPropElasticShotsGpu(w.elastic, w.par, *src, *rec)
    nl.setLanes(1)
    m = nl.modelSpace()
    m.getNdArray()[...] = w.source_signal()[None]
    out = nl.dataSpace()
    out.getNdArray()[...] = 0.0
    out.getNdArray().reshape(-1)[11] = np.inf
    nl.forward(True, m, out)                    # unchecked: succeeds and returns the Inf
    assert not np.isfinite(out.getNdArray()).all()
    _lib.check(nl._L.eio_ctx_set_check_finite(nl.ctx, 1))
    with pytest.raises(_lib.EioError) as e:
        nl.forward(True, m, out)
    assert e.value.code == -8
    fresh = nl.dataSpace()
    nl.forward(False, m, fresh)                 # finite again: no error
    assert np.isfinite(fresh.getNdArray()).all()
