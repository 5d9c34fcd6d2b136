"""Parity at the sizes of the benchmark configurations, against the CPU oracle.

* Born forward and adjoint on the full 600x1800 grid of the Born benchmark
  (900 receivers, the two of its ten shots nearest the middle of the line, the
  benchmark's smoothed 5 % perturbations), with
  the record shortened to nts = 300 so that the oracle finishes in seconds:
  FP32 engine vs FP32 oracle <= 1e-5, vs the FP64 oracle (elastic_iso_double
  semantics) <= 1e-4 relative L2.
* The FWI gradient of one cropped shot of the batched-FWI case (1000x3400
  grid, uneven 2-8 km receiver windows, smoothed start model, data from the
  true model), nts shortened to 400:
  - the gradient operator (the Born adjoint at the start model) applied to
    the FP64 oracle's residual: FP32 engine vs FP64 oracle <= 1e-4;
  - the whole gradient, residual formed in FP32 -- fused (the nonlinear forward
    records the source wavefield) and unfused (nonlinear forward, then the
    Born adjoint, the reference's composition): here the residual is under
    2 % of the data (the smoothed model reproduces the direct wave), so the
    FP32 rounding of the modelled data (6e-6 of it, the same in the FP32
    oracle, which follows the reference's float build) is amplified about
    60-fold.  Measured: engine 4.5e-4, FP32 oracle 2.3e-4 (the engine's fused
    taper and FMA-contracted stencils round differently).  Bound: within 3x of
    the FP32 oracle's own distance to FP64, and <= 1e-3;
  - with BF16 source-wavefield checkpoints: <= 2e-2 of the FP64 gradient.

The oracle runs on the cropped grid of the shot's window (the same pads, so the
same taper): a windowed shot equals the operator built on the cropped model.
"""
import numpy as np
import pytest

from elastic_isotropic_operators_b200 import prop, synthetic
from elastic_isotropic_operators_b200.sepvec import paramObj
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL32 = 1e-5
TOL64 = 1e-4
GRAD64 = 1e-4      # FP32 gradient vs the FP64 oracle's
BF16_GRAD64 = 2e-2  # BF16-checkpoint gradient vs the FP64 oracle's (stated, see the module docstring)


def test_born_full_600x1800_grid_vs_fp32_and_fp64_oracle():
    # shots 4 and 5 of the benchmark's ten lie inside the receiver spread
    w = synthetic.born_600x1800(nts=300, nshots=10, select=[4, 5])
    assert w.nExp == 2
    src, rec = w.geometry()
    sig = [w.source_signal()]
    born = prop.BornElasticShotsGpu(w.elastic, w.par, list(sig), *src, *rec)
    dm = born.modelSpace()
    dm.getNdArray()[...] = w.extra["dmodel"]
    d = born.dataSpace()
    born.forward(False, dm, d)
    c = O.Case.from_workload(w)
    f32, f64 = O.Oracle("f"), O.Oracle("d")
    fw32 = O.born_forward(f32, c, dm.getNdArray(), sig)
    fw64 = O.born_forward(f64, c, dm.getNdArray(), sig)
    got = d.getNdArray()
    assert np.abs(got).max() > 0
    e32, e64 = O.rel_l2(got, fw32), O.rel_l2(got, fw64)
    print("Born forward 600x1800: vs FP32 oracle %.3e, vs FP64 oracle %.3e" % (e32, e64))
    assert e32 < TOL32 and e64 < TOL64, (e32, e64)
    # adjoint of the FP64 forward data (a realistic data vector)
    dd = born.dataSpace()
    dd.getNdArray()[...] = fw64.astype(np.float32)
    g = born.modelSpace()
    born.adjoint(False, g, dd)
    ad32 = O.born_adjoint(f32, c, dd.getNdArray(), sig)
    ad64 = O.born_adjoint(f64, c, dd.getNdArray(), sig)
    a32, a64 = O.rel_l2(g.getNdArray(), ad32), O.rel_l2(g.getNdArray(), ad64)
    print("Born adjoint 600x1800: vs FP32 oracle %.3e, vs FP64 oracle %.3e" % (a32, a64))
    assert a32 < TOL32 and a64 < TOL64, (a32, a64)


def _cropped_case(w, elastic, ix0, nxw, rec_x):
    """Oracle case of one shot on grid columns [ix0, ix0 + nxw)."""
    ep = np.ascontiguousarray(np.asarray(elastic)[:, ix0:ix0 + nxw, :], np.float32)
    par = paramObj(w.par.as_dict())
    par.set("nx", str(nxw))
    par.set("nExp", "1")
    return O.Case(ep, par.as_dict(), w.oz, w.ox + ix0 * w.dx, [(w.src_z[:1], w.src_x[:1])],
                  (np.full(len(rec_x), w.rec_z[0], np.float32), np.asarray(rec_x, np.float32)))


def test_fwi_gradient_cropped_1000x3400_shot_vs_fp64_oracle():
    w = synthetic.fwi_1000x3400(nts=400, select=[37])
    src, rec = w.geometry()
    sig = w.source_signal()
    m_true = w.extra["true_model"]
    m0 = w.extra["start_model"]
    rec_x = w.extra["rec_x_shots"][0]

    born = prop.BornElasticShotsGpu(w.elastic, w.par, [sig], *src, *rec)
    ix0, nxw = born.autoShotWindows()
    ix0, nxw = int(ix0[0]), int(nxw[0])
    assert nxw < w.nx

    # observed data and the FP64 oracle gradient on the cropped grid; the FP32
    # oracle's gradient from the same observed data (the reference float arithmetic)
    f64, f32 = O.Oracle("d"), O.Oracle("f")
    c_true = _cropped_case(w, m_true, ix0, nxw, rec_x)
    c0 = _cropped_case(w, m0, ix0, nxw, rec_x)
    d_obs = O.nl_forward(f64, c_true, sig[None].astype(np.float64)).astype(np.float32)
    resid64 = O.nl_forward(f64, c0, sig[None].astype(np.float64)) - d_obs.astype(np.float64)
    assert np.abs(resid64).max() > 0
    phi64 = 0.5 * float(np.sum(resid64 * resid64))
    g64 = O.born_adjoint(f64, c0, resid64, [sig])
    resid32 = O.nl_forward(f32, c0, sig[None]) - d_obs
    g32_oracle = O.born_adjoint(f32, c0, resid32, [sig])
    e_oracle32 = O.rel_l2(g32_oracle, g64)

    def born_op(ckpt):
        b = prop.BornElasticShotsGpu(w.elastic, w.par, [sig], *src, *rec)
        b.setShotWindows([ix0], [nxw])
        b.setCheckpointPrecision(ckpt)
        return b

    def engine_gradient(fused, ckpt):
        b = born_op(ckpt)
        if fused:
            return b.fwiGradient(m0, sig[None], d_obs)
        nl = prop.nonlinearFwiPropElasticShotsGpu(w.elastic, w.par, sig[None], *src, *rec)
        nl.setShotWindows([ix0], [nxw])
        d = nl.dataSpace()
        nl.forward(False, m0, d)
        r = d.getNdArray() - d_obs
        b.setBackground(m0)
        g = b.modelSpace()
        rv = b.dataSpace()
        rv.getNdArray()[...] = r
        b.adjoint(False, g, rv)
        return 0.5 * float(np.sum(r.astype(np.float64) ** 2)), g.getNdArray()

    def inside(g, name):
        g = np.asarray(g)
        outside = np.concatenate([g[:, :ix0].ravel(), g[:, ix0 + nxw:].ravel()])
        assert not outside.any(), name           # the image stays inside the shot's window
        return g[:, ix0:ix0 + nxw]

    # the gradient operator on the FP64 residual
    b = born_op(0)
    b.setBackground(m0)
    g = b.modelSpace()
    rv = b.dataSpace()
    rv.getNdArray()[...] = resid64.astype(np.float32)
    b.adjoint(False, g, rv)
    e_op = O.rel_l2(inside(g.getNdArray(), "operator"), g64)

    results = {}
    for name, fused, ckpt in (("fused", True, 0), ("unfused", False, 0), ("fused-bf16", True, 1)):
        phi, g = engine_gradient(fused, ckpt)
        results[name] = (O.rel_l2(inside(g, name), g64), abs(phi - phi64) / phi64)
    print("FWI gradient 1000x3400 shot window %d+%d vs FP64 oracle: operator on the FP64 residual %.3e, "
          "FP32 oracle (reference float arithmetic) %.3e, engine (gradient, misfit) %s"
          % (ix0, nxw, e_op, e_oracle32, results))
    assert e_op < GRAD64, e_op
    bound = min(1e-3, max(GRAD64, 3.0 * e_oracle32))
    assert results["fused"][0] < bound and results["unfused"][0] < bound, (results, e_oracle32)
    assert results["fused-bf16"][0] < BF16_GRAD64, results
