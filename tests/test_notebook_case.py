"""The reference's own example case: notebooks/EFWI_test.p with the layered
VpVsRho models notebooks/true_layers.H and smooth_layers.H (101 x 201 cells,
10 m), 21 shots and 201 receivers at 510 m depth, sub = 4.

The models and the parameter file come from tests/golden/notebook_layers.npz
(written by tests/golden/make_notebook_case.py with the product's own SEP
reader).  CPU tests pin that fixture to the reference's files when the
reference tree is present, and check that the padding tool reproduces the pads
the parameter file carries (padElasticFileGpuMain's output for zPad = xPad =
100: zPadPlus 103, xPadPlus 115, a 312 x 424 grid).  The GPU tests run the
nonlinear forward (true model) and the Born adjoint (smooth model, residual
data) of all 21 shots, with the record shortened to nts = 100 (792 fine
steps), through the operator API built from the parameter file, and compare
them with the reference's own CUDA build (oracle/_ref) driven by the oracle's
host preparation: relative L2 <= 1e-5.
"""
import json
import os

import numpy as np
import pytest

from elastic_isotropic_operators_b200 import fwi, padding, prop
from elastic_isotropic_operators_b200.sepvec import axis, floatVector, hypercube, paramObj
from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURE = os.path.join(HERE, "golden", "notebook_layers.npz")
TREE = os.environ.get("EIO_REFERENCE_TREE", "/root/reference/elastic_iso_lib")
TOL32 = 1e-5


def _load():
    z = np.load(FIXTURE)
    par = json.loads(str(z["par"]))
    return z, par


def _model(z, name):
    ax = z[name + "_axes"]
    h = hypercube(axes=[axis(int(n), o, d) for n, o, d in ax])
    return floatVector(h, np.array(z[name], np.float32))


@pytest.mark.skipif(not os.path.isdir(os.path.join(TREE, "notebooks")), reason="reference tree not present")
def test_fixture_matches_the_reference_files():
    import importlib.util
    spec = importlib.util.spec_from_file_location("mk", os.path.join(HERE, "golden", "make_notebook_case.py"))
    mk = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mk)
    fresh = mk.read_case(TREE)
    z, par = _load()
    for k in ("true_layers", "smooth_layers", "true_layers_axes", "smooth_layers_axes"):
        np.testing.assert_array_equal(fresh[k], z[k])
    assert json.loads(str(fresh["par"])) == par


def test_padding_reproduces_the_parameter_file():
    z, par = _load()
    for name in ("true_layers", "smooth_layers"):
        v = _model(z, name)
        assert v.getNdArray().shape == (3, 201, 101)
        padded, pads = padding.padElasticFile(v, int(par["zPadMinus"]), int(par["xPadMinus"]))
        for k in ("zPadMinus", "zPadPlus", "xPadMinus", "xPadPlus"):
            assert pads[k] == int(par[k]), (k, pads[k], par[k])
        h = padded.getHyper()
        assert (h.getAxis(1).n, h.getAxis(2).n) == (int(par["nz"]), int(par["nx"]))
        assert h.getAxis(1).o == -(4 + 100) * 10.0 and h.getAxis(2).o == -(4 + 100) * 10.0
    # the layered model has 2-3 distinct values per parameter and the VpVsRho ranges of the notebook
    t = z["true_layers"]
    assert 1800.0 <= t[0].min() and t[0].max() <= 2200.0 and 1300.0 <= t[1].min() and t[1].max() <= 1600.0


def case(nts=100, nexp=None):
    """(par, elastic true, elastic smooth, oracle cases, source signal) of the
    notebook case, with nts coarse samples (and the first nexp shots)."""
    z, par = _load()
    par = dict(par)
    par["nts"] = str(nts)
    if nexp is not None:
        par["nExp"] = str(nexp)
    out = []
    for name in ("true_layers", "smooth_layers"):
        padded, _ = padding.padElasticFile(_model(z, name), int(par["zPadMinus"]), int(par["xPadMinus"]))
        ep = np.zeros_like(padded.getNdArray())
        fwi.ElasticConv(int(par["mod_par"])).forward(False, padded.getNdArray(), ep)   # VpVsRho -> rho, lambda, mu
        out.append(floatVector(padded.getHyper(), ep))
    p = paramObj(par)
    dts = p.getFloat("dts")
    from elastic_isotropic_operators_b200.wavelet import ricker_wavelet
    wav = ricker_wavelet(nts, dts, 8.0, 0.12).astype(np.float32)
    sig = np.zeros((5, 1, nts), np.float32)
    sig[2, 0] = wav
    sig[3, 0] = wav
    # the oracle's geometry: coordinates from the parameter file as the reference's
    # buildSourceGeometry / buildReceiversGeometry form them
    # (python_float/Elastic_iso_float_prop.py:205-364, 525-661): 1-based sample
    # indices of the unpadded model, plus the top/left pad and the fat frame
    h = out[0].getHyper()
    oz, dz, ox, dx = h.getAxis(1).o, h.getAxis(1).d, h.getAxis(2).o, h.getAxis(2).d
    fat = 4
    zs = p.getInt("zSource") - 1 + p.getInt("zPadMinus") + fat
    xs = p.getInt("xSource") - 1 + p.getInt("xPadMinus") + fat
    src = [(np.array([oz + zs * dz], np.float32), np.array([ox + (xs + e * p.getInt("spacingShots")) * dx],
                                                           np.float32)) for e in range(p.getInt("nExp"))]
    zr = p.getInt("depthReceiver") - 1 + p.getInt("zPadMinus") + fat
    xr = p.getInt("oReceiver") - 1 + p.getInt("xPadMinus") + fat
    nr = p.getInt("nReceiver")
    rec = (np.full(nr, oz + zr * dz, np.float32),
           np.array([ox + (xr + i * p.getInt("dReceiver")) * dx for i in range(nr)], np.float32))
    cases = [O.Case(v.getNdArray(), par, oz, ox, src, rec) for v in out]
    return p, out[0], out[1], cases, sig


@pytest.mark.gpu
@pytest.mark.skipif(not O.RefGpu.available("f"), reason="oracle/_ref not built")
def test_notebook_case_matches_the_reference_cuda_build():
    p, true_el, smooth_el, (c_true, c_smooth), sig = case()
    src = prop.buildSourceGeometry(p, true_el)[:4]
    rec = prop.buildReceiversGeometry(p, true_el)[:4]
    ref = O.RefGpu("f")
    orc = O.Oracle("f")

    # nonlinear forward on the true model, all 21 shots
    nl = prop.nonlinearPropElasticShotsGpu(true_el, p, *src, *rec)
    model = nl.modelSpace()
    model.getNdArray()[...] = sig[None]
    d_true = nl.dataSpace()
    nl.forward(False, model, d_true)
    assert d_true.getNdArray().shape == (21, 5, 201, 100)
    want = O.nl_forward(orc, c_true, model.getNdArray(), engine=ref)
    err_nl = O.rel_l2(d_true.getNdArray(), want)
    assert np.abs(want).max() > 0
    print("notebook case, nonlinear forward vs reference CUDA build: %.3e" % err_nl)
    assert err_nl < TOL32, err_nl

    # Born adjoint at the smooth model of the true-minus-smooth data
    nl.setBackground(smooth_el)
    d_smooth = nl.dataSpace()
    nl.forward(False, model, d_smooth)
    resid = d_true.getNdArray() - d_smooth.getNdArray()
    assert np.abs(resid).max() > 0
    born = prop.BornElasticShotsGpu(smooth_el, p, [sig], *src, *rec)
    g = born.modelSpace()
    dv = born.dataSpace()
    dv.getNdArray()[...] = resid
    born.adjoint(False, g, dv)
    gwant = O.born_adjoint(orc, c_smooth, resid, [sig], engine=ref)
    err_born = O.rel_l2(g.getNdArray(), gwant)
    print("notebook case, Born adjoint vs reference CUDA build: %.3e" % err_born)
    assert err_born < TOL32, err_born
