"""Shot batching of the nonlinear forward and adjoint (eio_ctx_set_shot_batch):
up to 8 shots advanced in lockstep with one step launch for all of them.

With the tile kernel pinned on both sides, the batched traces equal the
one-shot-at-a-time (lanes) traces bit for bit: same stencil body, same time
weights, each shot on its own point lists and window.  With the autotuned
kernel on the unbatched side, they agree to 1e-6 (relative L2)."""
import numpy as np
import pytest

from elastic_isotropic_operators_b200 import _lib, prop, synthetic
from elastic_isotropic_operators_b200._lib import EioError

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a, b = np.ravel(a).astype(np.float64), np.ravel(b).astype(np.float64)
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def _forward(w, batch, pin, windows=False, add=False, base=None):
    src, rec = w.geometry()
    op = prop.nonlinearPropElasticShotsGpu(w.elastic, w.par, *src, *rec)
    if pin:
        _lib.check(op._L.eio_ctx_set_kernel(op.ctx, 0, 64, 16, 2))
    if windows:
        op.autoShotWindows()
    op.setShotBatch(batch)
    model = op.modelSpace()
    model.getNdArray()[...] = w.source_signal()[None]
    data = op.dataSpace()
    if base is not None:
        data.getNdArray()[...] = base
    op.forward(add, model, data)
    return data.getNdArray().copy()


@pytest.mark.parametrize("batch", [2, 4, 8])
def test_batched_forward_equals_one_shot_at_a_time(batch):
    w = synthetic.small(nts=150, nshots=5)
    ref = _forward(w, 1, True)
    out = _forward(w, batch, True)
    assert np.array_equal(out, ref)
    auto = _forward(w, 1, False)
    assert _rel(out, auto) < 1e-6


def test_batched_forward_with_cropped_shots_and_add():
    w = synthetic.fwi_1000x3400(nz=136, nx=520, nts=300, nshots=6, nrec=30, pad=20, window_km=(1.0, 2.5))
    ref = _forward(w, 1, True, windows=True)
    out = _forward(w, 4, True, windows=True)
    assert np.array_equal(out, ref)
    base = np.random.default_rng(0).standard_normal(ref.shape).astype(np.float32)
    acc = _forward(w, 4, True, windows=True, add=True, base=base)
    assert np.array_equal(acc, base + ref)


def test_batch_size_is_checked():
    w = synthetic.small(nts=60, nshots=1)
    src, rec = w.geometry()
    op = prop.nonlinearPropElasticShotsGpu(w.elastic, w.par, *src, *rec)
    for bad in (0, 9):
        with pytest.raises(EioError):
            op.setShotBatch(bad)


def _adjoint(w, batch, pin, nme, windows=False, lanes=1):
    src, rec = w.geometry()
    op = prop.nonlinearPropElasticShotsGpu(w.elastic, w.par, *src, *rec)
    if pin:
        _lib.check(op._L.eio_ctx_set_kernel(op.ctx, 0, 64, 16, 2))
    _lib.check(op._L.eio_ctx_set_lanes(op.ctx, lanes))
    if windows:
        op.autoShotWindows()
    op.setShotBatch(batch)
    data = op.dataSpace()
    data.getNdArray()[...] = np.random.default_rng(3).standard_normal(data.getNdArray().shape).astype(np.float32)
    model = np.zeros((nme, 5, op.nSrcIrreg, w.nts), np.float32)
    op.adjoint(False, model, data)
    return model


@pytest.mark.parametrize("nme", [1, 5])
def test_batched_adjoint_equals_one_shot_at_a_time(nme):
    w = synthetic.small(nts=150, nshots=5)
    ref = _adjoint(w, 1, True, nme)
    out = _adjoint(w, 4, True, nme)
    assert np.array_equal(out, ref)          # shots stacked in the same order
    auto = _adjoint(w, 1, False, nme, lanes=2)
    assert _rel(out, auto) < 1e-6


def test_batched_adjoint_with_cropped_shots():
    w = synthetic.fwi_1000x3400(nz=136, nx=520, nts=300, nshots=6, nrec=30, pad=20, window_km=(1.0, 2.5))
    ref = _adjoint(w, 1, True, 6, windows=True)
    out = _adjoint(w, 8, True, 6, windows=True)
    assert np.array_equal(out, ref)
