"""Cropped shots (eio_ctx_set_shot_windows): every shot of a multi-shot call
propagates on its own window of the grid.

A shot on its window must equal the same shot propagated by an operator built
on the cropped model (same pads, so the same cosine taper): nonlinear traces,
Born traces and the Born image on the window's interior (relative L2 <= 1e-5,
the same arithmetic on the same values).  The windowed operators stay exact
adjoints (dot tests), devices outside a window are rejected, and the automatic
windows hold each shot's aperture."""
import numpy as np
import pytest

from elastic_isotropic_operators_b200 import _lib, prop, synthetic
from elastic_isotropic_operators_b200.prop import EioError, _staggered_hypers, spaceInterpGpu
from elastic_isotropic_operators_b200.sepvec import paramObj

pytestmark = pytest.mark.gpu

FAT = 4


def _case():
    """232-column grid, two shots with uneven receiver apertures."""
    w = synthetic.small(nz=72, nx=232, nts=70, nshots=2)
    dx, ox = w.dx, w.ox
    col = lambda ix: np.float32(ox + ix * dx)
    # off-grid by binary-exact fractions, so that the cropped operators (another x
    # origin) compute the same interpolation weights
    src_x = [col(60) + np.float32(2.5), col(160) + np.float32(7.5)]
    # the data vector is rectangular: the same device count, different extents
    recs = [np.linspace(44, 95, 18).astype(int), np.linspace(120, 188, 18).astype(int)]
    return w, src_x, recs


def _geometry(w, elastic, src_x, recs, shots):
    hyps = _staggered_hypers(elastic)
    src = [[], [], [], []]
    rec = [[], [], [], []]
    for e in shots:
        zc = w.src_z[e:e + 1].copy()
        xc = np.array([src_x[e]], np.float32)
        rx = np.array([w.ox + ix * w.dx + 2.5 for ix in recs[e]], np.float32)
        rz = np.full(rx.size, w.rec_z[0], np.float32)
        for k, h in enumerate(hyps):
            src[k].append(spaceInterpGpu(zc, xc, h, w.nts, "linear", 1, 0, 0.0, 0.0))
            rec[k].append(spaceInterpGpu(rz, rx, h, w.nts, "linear", 1, 0, 0.0, 0.0))
    return src, rec


def _cropped(w, ix0, nxw):
    ep = np.array(w.elastic.getNdArray())[:, ix0:ix0 + nxw, :].copy()
    el = synthetic.elastic_vector(ep, w.oz, w.ox + ix0 * w.dx, w.dz, w.dx)
    par = paramObj(w.par.as_dict())
    par.set("nx", str(nxw))
    par.set("nExp", "1")
    return el, par


def _full_ops(w, src_x, recs):
    src, rec = _geometry(w, w.elastic, src_x, recs, [0, 1])
    nl = prop.nonlinearPropElasticShotsGpu(w.elastic, w.par, *src, *rec)
    born = prop.BornElasticShotsGpu(w.elastic, w.par, [w.source_signal()], *src, *rec)
    return nl, born


def _rel(a, b):
    a, b = np.ravel(a).astype(np.float64), np.ravel(b).astype(np.float64)
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("kind", [3, 5])
def test_windowed_shots_equal_cropped_operators(kind):
    w, src_x, recs = _case()
    nl, born = _full_ops(w, src_x, recs)
    for op in (nl, born):
        op.setShotWindows([24, 104], [88, 120])
        _lib.check(op._L.eio_ctx_set_kernel(op.ctx, kind, 64, 16, 0))
    rng = np.random.default_rng(3)
    model = nl.modelSpace()
    model.getNdArray()[...] = w.source_signal()[None]
    data = nl.dataSpace()
    nl.forward(False, model, data)
    dm = born.modelSpace()
    dm.getNdArray()[...] = rng.standard_normal(dm.getNdArray().shape).astype(np.float32) * 1e-3
    bdata = born.dataSpace()
    born.forward(False, dm, bdata)
    resid = born.dataSpace()
    resid.getNdArray()[...] = rng.standard_normal(resid.getNdArray().shape).astype(np.float32)
    for e, (ix0, nxw) in enumerate([(24, 88), (104, 120)]):
        el, par = _cropped(w, ix0, nxw)
        src, rec = _geometry(w, el, src_x, recs, [e])
        nl_c = prop.nonlinearPropElasticShotsGpu(el, par, *src, *rec)
        _lib.check(nl_c._L.eio_ctx_set_kernel(nl_c.ctx, kind, 64, 16, 0))   # the same kernel, the same sums
        d_c = nl_c.dataSpace()
        nl_c.forward(False, model, d_c)
        assert _rel(data.getNdArray()[e], d_c.getNdArray()[0]) < 1e-5, ("nl", e)
        born_c = prop.BornElasticShotsGpu(el, par, [w.source_signal()], *src, *rec)
        _lib.check(born_c._L.eio_ctx_set_kernel(born_c.ctx, kind, 64, 16, 0))
        dm_c = born_c.modelSpace()
        dm_c.getNdArray()[...] = dm.getNdArray()[:, ix0:ix0 + nxw, :]
        bd_c = born_c.dataSpace()
        born_c.forward(False, dm_c, bd_c)
        assert _rel(bdata.getNdArray()[e], bd_c.getNdArray()[0]) < 1e-5, ("born fwd", e)
        # the image of this shot alone, compared away from the window's frame
        r1 = born.dataSpace()
        r1.getNdArray()[e] = resid.getNdArray()[e]
        g = born.modelSpace()
        born.adjoint(False, g, r1)
        rc = born_c.dataSpace()
        rc.getNdArray()[0] = resid.getNdArray()[e]
        g_c = born_c.modelSpace()
        born_c.adjoint(False, g_c, rc)
        inner = slice(FAT + 1, nxw - FAT - 1)
        got = g.getNdArray()[:, ix0:ix0 + nxw, :][:, inner, :]
        want = g_c.getNdArray()[:, inner, :]
        assert _rel(got, want) < 1e-5, ("born adj", e)
        outside = np.ones(w.nx, bool)
        outside[ix0:ix0 + nxw] = False
        assert np.abs(g.getNdArray()[:, outside, :]).max() == 0.0


def test_windowed_operators_are_adjoints_and_auto_windows():
    w, src_x, recs = _case()
    nl, born = _full_ops(w, src_x, recs)
    ix0, nxw = born.autoShotWindows(margin=12)
    for e in range(2):
        assert (nxw[e] - 2 * FAT) % 16 == 0 and 0 <= ix0[e] and ix0[e] + nxw[e] <= w.nx
        assert ix0[e] + FAT <= min(recs[e].min(), 60 if e == 0 else 160) - 12
        assert ix0[e] + nxw[e] - FAT > max(recs[e].max(), 60 if e == 0 else 160) + 12
        assert nxw[e] < w.nx
    assert born.dotTest(False, 1e-5), born.lastDotTest
    nl.autoShotWindows(margin=12)
    assert nl.dotTest(False, 1e-5), nl.lastDotTest
    nl.clearShotWindows()
    assert nl.dotTest(False, 1e-5), nl.lastDotTest


def test_device_outside_window_is_rejected():
    w, src_x, recs = _case()
    nl, _ = _full_ops(w, src_x, recs)
    nl.setShotWindows([24, 24], [88, 88])      # shot 1 lies far outside [24, 112)
    model = nl.modelSpace()
    model.getNdArray()[...] = w.source_signal()[None]
    with pytest.raises(EioError):
        nl.forward(False, model, nl.dataSpace())
    with pytest.raises(EioError):
        nl.setShotWindows([24, 104], [90, 120])  # 90 - 8 is not a multiple of 16
