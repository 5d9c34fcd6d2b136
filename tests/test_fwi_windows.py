"""The batched-FWI configuration (1000x3400 grid, uneven 2-8 km receiver
windows, cropped shots, BF16 source-wavefield checkpoints, shot lanes).

* At full size (one shot, nts = 5000): the cropped, BF16-checkpointed Born
  operator is an exact adjoint (FP64 dot test <= 1e-5).
* On a reduced grid with several shots: the FWI gradient with cropped shots
  and BF16 checkpoints stays within 2e-2 (relative L2) of the same gradient
  with FP32 checkpoints, and cropping keeps the direction of the whole-grid
  gradient (cosine >= 0.9)."""
import numpy as np
import pytest

from elastic_isotropic_operators_b200 import fwi, prop, synthetic

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a, b = np.ravel(a).astype(np.float64), np.ravel(b).astype(np.float64)
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def test_full_size_windowed_bf16_born_dot_test():
    w = synthetic.fwi_1000x3400(nshots=1)
    src, rec = w.geometry()
    born = prop.BornElasticShotsGpu(w.elastic, w.par, [w.source_signal()], *src, *rec)
    born.setCheckpointPrecision(1)
    ix0, nxw = born.autoShotWindows()
    assert nxw[0] < w.nx
    span = w.extra["rec_x_shots"][0]
    assert span.max() - span.min() >= 2000.0 - 2 * w.dx
    assert born.dotTest(False, 1e-5), born.lastDotTest


def _objective(w, d_obs, windows, ckpt):
    src, rec = w.geometry()
    sig = w.source_signal()[None]
    nl = prop.nonlinearFwiPropElasticShotsGpu(w.elastic, w.par, sig, *src, *rec)
    born = prop.BornElasticShotsGpu(w.elastic, w.par, [w.source_signal()], *src, *rec)
    born.setCheckpointPrecision(ckpt)
    if windows:
        nl.autoShotWindows()
        born.autoShotWindows()
    return fwi.FwiObjective(nl, born, d_obs)


def test_gradient_with_cropped_shots_and_bf16_checkpoints():
    w = synthetic.fwi_1000x3400(nz=136, nx=520, nts=600, nshots=4, nrec=40, pad=20, window_km=(1.0, 2.5))
    src, rec = w.geometry()
    sig = w.source_signal()[None]
    true_op = prop.nonlinearFwiPropElasticShotsGpu(w.elastic, w.par, sig, *src, *rec)
    d_obs = true_op.dataSpace()
    true_op.forward(False, w.extra["true_model"], d_obs)
    m0 = w.extra["start_model"]
    _, g_full = _objective(w, d_obs, False, 0).value_and_gradient(m0)
    phi32, g32 = _objective(w, d_obs, True, 0).value_and_gradient(m0)
    phi16, g16 = _objective(w, d_obs, True, 1).value_and_gradient(m0)
    assert phi32 > 0 and abs(phi16 - phi32) <= 1e-6 * phi32   # the misfit does not use the history
    assert _rel(g16, g32) < 2e-2, _rel(g16, g32)
    a, b = np.ravel(g32).astype(np.float64), np.ravel(g_full).astype(np.float64)
    cos = a @ b / (np.linalg.norm(a) * np.linalg.norm(b))
    assert cos >= 0.9, cos
