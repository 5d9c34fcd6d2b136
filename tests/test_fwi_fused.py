"""The fused FWI gradient (BornElasticShotsGpu.fwiGradient, eio_fwi_gradient):
per shot, the nonlinear forward records the Born source wavefield, and the
Born adjoint of the residual runs on that recording.

The unfused evaluation (nonlinear forward, then the Born adjoint, which
propagates the source again) is the reference: the two inject the same source
signal through different roundings (coarse traces with the time filter in the
nonlinear step, host-interpolated fine traces in the Born step), so misfit,
modelled data and gradient agree to FP32 rounding, not bitwise.  Bounds: the
modelled data and the misfit to 1e-5 relative, the gradient to 1e-4 relative
L2 (FP32 history), 2e-2 with BF16 history (the quantisation of the history
itself, as for the unfused path)."""
import numpy as np
import pytest

from elastic_isotropic_operators_b200 import fwi, prop, synthetic
from elastic_isotropic_operators_b200._lib import EioError

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a, b = np.ravel(a).astype(np.float64), np.ravel(b).astype(np.float64)
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def _ops(w, lanes=None, ckpt=0):
    src, rec = w.geometry()
    sig = w.source_signal()
    nl = prop.nonlinearFwiPropElasticShotsGpu(w.elastic, w.par, sig[None], *src, *rec)
    born = prop.BornElasticShotsGpu(w.elastic, w.par, [sig], *src, *rec)
    born.setCheckpointPrecision(ckpt)
    if lanes is not None:
        born.setLanes(lanes)
    return nl, born


def _observed(w, nl, model, sampler=None):
    d = nl.dataSpace()
    nl.forward(False, model, d)
    d = d.getNdArray().copy()
    if sampler is not None:
        ds = np.zeros(sampler.range_shape(d.shape), np.float32)
        sampler.forward(False, d, ds)
        d = ds
    return d


def _start(true):
    nx, nz = true.shape[1], true.shape[2]
    xx, zz = np.meshgrid(np.arange(nx), np.arange(nz), indexing="ij")
    blob = np.exp(-((xx - nx / 2) ** 2 + (zz - nz / 2) ** 2) / (2 * 8.0 ** 2)).astype(np.float32)
    m0 = true.copy()
    m0[1] *= 1 - 0.04 * blob
    m0[2] *= 1 - 0.04 * blob
    return m0


@pytest.mark.parametrize("lanes", [1, 2])
@pytest.mark.parametrize("components", [None, "p,vx,vz"])
def test_fused_gradient_matches_unfused(lanes, components):
    w = synthetic.small(nts=140, nshots=3)
    nl, born = _ops(w, lanes)
    true = w.elastic.getNdArray().copy()
    S = None if components is None else fwi.ElasticDatComp(components)
    d_obs = _observed(w, nl, true, S)
    m0 = _start(true)
    phi_u, g_u = fwi.FwiObjective(nl, born, d_obs, sampler=S, fused=False).value_and_gradient(m0)
    data = np.zeros(nl.dataSpace().getNdArray().shape, np.float32)
    phi_f, g_f = born.fwiGradient(m0, nl.sources, d_obs, components, data=data)
    assert phi_u > 0 and abs(phi_f - phi_u) <= 1e-5 * phi_u, (phi_f, phi_u)
    d_ref = _observed(w, nl, m0)
    assert _rel(data, d_ref) < 1e-5, _rel(data, d_ref)
    assert _rel(g_f, g_u) < 1e-4, _rel(g_f, g_u)
    # FwiObjective takes the fused path by default
    obj = fwi.FwiObjective(nl, born, d_obs, sampler=S)
    assert obj.fused
    phi_o, g_o = obj.value_and_gradient(m0)
    assert phi_o == phi_f and np.array_equal(g_o, g_f)


def test_fused_gradient_lane_count_does_not_change_the_result_beyond_summation_order():
    w = synthetic.small(nts=120, nshots=4)
    true = w.elastic.getNdArray().copy()
    nl, born1 = _ops(w, 1)
    d_obs = _observed(w, nl, true)
    m0 = _start(true)
    phi1, g1 = born1.fwiGradient(m0, nl.sources, d_obs)
    _, born2 = _ops(w, 2)
    phi2, g2 = born2.fwiGradient(m0, nl.sources, d_obs)
    assert phi1 == phi2                      # per-shot misfits summed in shot order
    assert _rel(g2, g1) < 1e-6, _rel(g2, g1)


def test_fused_gradient_with_cropped_shots_and_bf16_history():
    w = synthetic.fwi_1000x3400(nz=136, nx=520, nts=600, nshots=4, nrec=40, pad=20, window_km=(1.0, 2.5))
    src, rec = w.geometry()
    sig = w.source_signal()
    nl = prop.nonlinearFwiPropElasticShotsGpu(w.elastic, w.par, sig[None], *src, *rec)
    d_obs = _observed(w, nl, w.extra["true_model"])
    m0 = w.extra["start_model"]
    res = {}
    for ckpt in (0, 1):
        born = prop.BornElasticShotsGpu(w.elastic, w.par, [sig], *src, *rec)
        born.setCheckpointPrecision(ckpt)
        born.autoShotWindows()
        nl.autoShotWindows()
        res[ckpt] = (fwi.FwiObjective(nl, born, d_obs, fused=False).value_and_gradient(m0),
                     born.fwiGradient(m0, nl.sources, d_obs))
    (phi_u, g_u), (phi_f, g_f) = res[0]
    assert abs(phi_f - phi_u) <= 1e-5 * phi_u
    assert _rel(g_f, g_u) < 1e-4, _rel(g_f, g_u)
    (_, g_u16), (phi_f16, g_f16) = res[1]
    assert phi_f16 == phi_f                  # the misfit does not use the history
    assert _rel(g_f16, g_u16) < 2e-2 and _rel(g_f16, g_f) < 2e-2


def test_fused_gradient_rejects_bad_arguments():
    w = synthetic.small(nts=80, nshots=1)
    nl, born = _ops(w)
    d_obs = np.zeros((1, 2, born.nRecIrreg, w.nts), np.float32)
    with pytest.raises(EioError):
        born.fwiGradient(w.elastic.getNdArray(), nl.sources, d_obs, "vx,vx")
    with pytest.raises(EioError):
        born.fwiGradient(w.elastic.getNdArray(), nl.sources, d_obs, "vx,vz,p")   # dObs holds 2 components
    ws = synthetic.small(nts=80, nshots=1, surface=1)
    nls, borns = _ops(ws)
    assert not fwi.FwiObjective(nls, borns, d_obs).fused
    with pytest.raises(EioError):
        borns.fwiGradient(ws.elastic.getNdArray(), nls.sources, np.zeros((1, 5, borns.nRecIrreg, ws.nts),
                                                                           np.float32))
