"""FWI objective and L-BFGS on the GPU operators (small layered case).

The gradient is the Born adjoint of the residual, the reference's choice; the
reference's Born operator matches the derivative of the nonlinear operator to
about 1 % (its coarse-time secondary source), hence the 5 % bound below."""
import numpy as np
import pytest

from elastic_isotropic_operators_b200 import fwi, prop, synthetic

pytestmark = pytest.mark.gpu


def _problem(sampler=None, mask=None):
    w = synthetic.small(nts=120)
    src, rec = w.geometry()
    sig = w.source_signal()
    true = w.elastic.getNdArray().copy()
    nl = prop.nonlinearFwiPropElasticShotsGpu(w.elastic, w.par, sig[None], *src, *rec)
    born = prop.BornElasticShotsGpu(w.elastic, w.par, [sig], *src, *rec)
    d = nl.dataSpace()
    nl.forward(False, true, d)
    d_obs = d.getNdArray().copy()
    if sampler is not None:
        ds = np.zeros(sampler.range_shape(d_obs.shape), np.float32)
        sampler.forward(False, d_obs, ds)
        d_obs = ds
    # start model: lambda and mu lowered by up to 4 % in a smooth blob
    nx, nz = true.shape[1], true.shape[2]
    xx, zz = np.meshgrid(np.arange(nx), np.arange(nz), indexing="ij")
    blob = np.exp(-((xx - nx / 2) ** 2 + (zz - nz / 2) ** 2) / (2 * 8.0 ** 2)).astype(np.float32)
    m0 = true.copy()
    m0[1] *= 1 - 0.04 * blob
    m0[2] *= 1 - 0.04 * blob
    return fwi.FwiObjective(nl, born, d_obs, sampler=sampler, mask=mask), m0, true


def test_gradient_matches_central_difference():
    obj, m0, _ = _problem()
    phi, g = obj.value_and_gradient(m0)
    assert phi > 0 and np.isfinite(g).all()
    rng = np.random.default_rng(4)
    dm = synthetic.gaussian_smooth(rng.standard_normal(m0.shape[1:]), 3.0).astype(np.float32)
    dm = np.stack([dm * 0.0, dm, dm]) * (0.01 * m0 / np.abs(dm).max())
    h = 0.5
    fd = (obj.value(m0 + h * dm) - obj.value(m0 - h * dm)) / (2 * h)
    gd = fwi.dot64(g, dm)
    assert abs(fd - gd) < 0.05 * abs(fd), (fd, gd)


def test_lbfgs_reduces_the_misfit_with_bounds_mask_and_components():
    S = fwi.ElasticDatComp("p,vx,vz")
    obj, m0, true = _problem()
    mask = np.ones_like(m0)
    mask[:, :, :12] = 0.0                      # freeze the top rows
    obj_s, _, _ = _problem(sampler=S, mask=mask)
    lo, hi = m0 * 0.9, m0 * 1.1
    m, hist = fwi.lbfgs(obj_s, m0, niter=3, minBound=lo, maxBound=hi, scale=m0)
    assert len(hist) == 4
    assert all(b < a for a, b in zip(hist, hist[1:]))
    assert hist[-1] < 0.8 * hist[0]
    assert (m >= lo - 1e-5 * np.abs(lo)).all() and (m <= hi + 1e-5 * np.abs(hi)).all()
    assert np.allclose(m[:, :, :12], m0[:, :, :12], rtol=1e-6)
    # the update moves lambda and mu towards the true model
    err0 = np.linalg.norm((m0 - true)[1:])
    err1 = np.linalg.norm((m - true)[1:])
    assert err1 < err0


def test_multiscale_bands_reduce_the_misfit_of_each_band():
    from elastic_isotropic_operators_b200 import wavelet
    w = synthetic.small(nts=120)
    src, rec = w.geometry()
    sig = w.source_signal()
    true = w.elastic.getNdArray().copy()
    nl = prop.nonlinearFwiPropElasticShotsGpu(w.elastic, w.par, sig[None], *src, *rec)
    born = prop.BornElasticShotsGpu(w.elastic, w.par, [sig], *src, *rec)
    d = nl.dataSpace()
    nl.forward(False, true, d)
    d_obs = d.getNdArray().copy()
    _, m0, _ = _problem()
    sources = nl.sources.copy()
    bands = wavelet.multiscale_bands(4.0, 20.0, 2, ramp=2.0)
    m, hists = fwi.multiscale(lambda band: fwi.band_objective(nl, born, d_obs, sources, w.dts, band), m0, bands,
                              niter=2, scale=m0)
    assert len(hists) == 2
    assert all(h[-1] < h[0] for h in hists), hists
    # the Born operator took the band-limited signals
    assert not np.allclose(born._sigs[0], sig.reshape(born._sigs[0].shape))
