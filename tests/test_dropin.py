"""The drop-in modules (elastic_isotropic_operators_b200/dropin): the
reference's scripts import pyElastic_iso_float_nl, pyElastic_iso_float_born,
Elastic_iso_float_prop and SEP's Python stack by those names.

* CPU: the modules load under the reference's names; genericIO expands par
  files; when the reference tree is present, its own unmodified
  nonlinearPythonElasticFloatMain.py and BornPythonElasticFloatMain.py run
  (forward and adjoint, ``par=`` file, SEP files in and out) with the engine
  classes of the two pybind modules replaced by a test double that computes
  with the CPU oracle -- so this checks the scripts' whole host path (parameter
  handling, model conversion, geometry, vector shapes, file I/O) without a
  GPU, against the oracle run directly on the case.
* GPU: the same four runs through the drop-in set-up functions and operator
  wrappers in the scripts' order, on the real engine, against the oracle
  (relative L2 <= 1e-5).

The case is the reference's notebook case (EFWI_test.p, true_layers.H,
VpVsRho, sub = 4), shortened to two shots and nts = 60.
"""
import os
import runpy
import sys

import numpy as np
import pytest

from elastic_isotropic_operators_b200 import dropin, padding, sepio
from elastic_isotropic_operators_b200.sepvec import axis, floatVector, hypercube
from oracle import oracle as O

from test_notebook_case import TREE, _load, _model, case

SCRIPTS = os.path.join(TREE, "python", "python_float")
NTS, NEXP = 60, 2
TOL32 = 1e-5


def _modules():
    dropin.activate()
    import Elastic_iso_float_prop
    import genericIO
    import pyElastic_iso_float_born
    import pyElastic_iso_float_nl
    return Elastic_iso_float_prop, genericIO, pyElastic_iso_float_nl, pyElastic_iso_float_born


def test_dropin_modules_load_under_the_reference_names():
    P, G, NL, BORN = _modules()
    import Hypercube
    import SepVector
    import elasticParamConvertModule
    import pyDaskOperator
    import pyOperator
    for name in ("nonlinearOpInitFloat", "nonlinearFwiOpInitFloat", "BornOpInitFloat", "buildSourceGeometry",
                 "buildReceiversGeometry", "nonlinearPropElasticShotsGpu", "nonlinearFwiPropElasticShotsGpu",
                 "BornElasticShotsGpu", "create_client", "parfile2pars"):
        assert hasattr(P, name), name
    assert hasattr(NL, "spaceInterpGpu") and hasattr(NL, "nonlinearPropElasticShotsGpu")
    assert hasattr(NL, "ostream_redirect") and hasattr(BORN, "BornElasticShotsGpu")
    assert issubclass(P.BornElasticShotsGpu, pyOperator.Operator)
    assert Hypercube.axis(n=3).n == 3 and SepVector.getSepVector(ns=[4, 2]).getNdArray().shape == (2, 4)
    assert hasattr(elasticParamConvertModule, "ElasticConv")
    with pytest.raises(NotImplementedError):
        pyDaskOperator.DaskOperator(None, None, None, None)
    with pytest.raises(NotImplementedError):
        P.create_client(G.io(params=["x", "hostnames=a,b"]))
    assert P.create_client(G.io(params=["x"])) == (None, None)


def test_genericIO_expands_par_files(tmp_path):
    _, G, _, _ = _modules()
    pf = tmp_path / "p.p"
    pf.write_text("nts=750  #samples\ndts=0.004 sub=4\niGpu=0,1\n")
    par = G.io(params=["prog.py", "nz=7", "par=%s" % pf, "nts=60"])
    assert par.getInt("nts") == 60 and par.getFloat("dts") == 0.004 and par.getInt("sub") == 4
    assert par.getInt("nz") == 7 and par.getInts("iGpu") == [0, 1] and par.getInt("adj", 0) == 0
    assert par.getCpp().param is par


def _write_inputs(d):
    """SEP files and par file of the shortened notebook case (VpVsRho model)."""
    z, par = _load()
    padded, _ = padding.padElasticFile(_model(z, "true_layers"), int(par["zPadMinus"]), int(par["xPadMinus"]))
    padded.writeVec(str(d / "vpvsrho.H"))
    smooth, _ = padding.padElasticFile(_model(z, "smooth_layers"), int(par["zPadMinus"]), int(par["xPadMinus"]))
    smooth.writeVec(str(d / "smooth.H"))
    p, true_el, smooth_el, (c_true, c_smooth), sig = case(NTS, NEXP)
    lines = ["%s=%s" % (k, v) for k, v in p.as_dict().items() if k != "iGpu"]
    (d / "case.p").write_text("\n".join(lines) + "\n")
    t = axis(NTS, 0.0, p.getFloat("dts"))
    floatVector(hypercube(axes=[t, axis(5)]), sig[:, 0, :]).writeVec(str(d / "wavelet.H"))
    floatVector(hypercube(axes=[t, axis(1), axis(5)]), sig).writeVec(str(d / "sources.H"))
    rng = np.random.default_rng(4)
    dm = (rng.standard_normal((3,) + true_el.getNdArray().shape[1:]) *
          np.array([10.0, 1e7, 1e7])[:, None, None]).astype(np.float32)
    floatVector(true_el.getHyper(), dm).writeVec(str(d / "dmodel.H"))
    return p, true_el, smooth_el, c_true, c_smooth, sig, dm


class _OracleNl:
    """Test double of pyElastic_iso_float_nl.nonlinearPropElasticShotsGpu:
    the same constructor and methods, computed by the CPU oracle."""

    def __init__(self, elasticParam, par, sC, sX, sZ, sXZ, rC, rX, rZ, rXZ):
        h = elasticParam.getHyper()
        self.case = O.Case(np.array(elasticParam.getNdArray()), par.as_dict(), h.getAxis(1).o, h.getAxis(2).o,
                           [(g.zCoord, g.xCoord) for g in sC], (rC[0].zCoord, rC[0].xCoord))

    def forward(self, add, model, data):
        out = O.nl_forward(O.Oracle("f"), self.case, model.getNdArray())
        data.getNdArray()[...] = out + (data.getNdArray() if add else 0.0)

    def adjoint(self, add, model, data):
        m = model.getNdArray()
        out = O.nl_adjoint(O.Oracle("f"), self.case, data.getNdArray(), nModelExp=m.shape[0])
        m[...] = out + (m if add else 0.0)


class _OracleBorn:
    """Test double of pyElastic_iso_float_born.BornElasticShotsGpu (CPU oracle)."""

    def __init__(self, elasticParam, par, signals, sC, sX, sZ, sXZ, rC, rX, rZ, rXZ):
        h = elasticParam.getHyper()
        self.sig = [np.array(s.getNdArray()) for s in signals]
        self.case = O.Case(np.array(elasticParam.getNdArray()), par.as_dict(), h.getAxis(1).o, h.getAxis(2).o,
                           [(g.zCoord, g.xCoord) for g in sC], (rC[0].zCoord, rC[0].xCoord))

    def forward(self, add, model, data):
        out = O.born_forward(O.Oracle("f"), self.case, model.getNdArray(), self.sig)
        data.getNdArray()[...] = out + (data.getNdArray() if add else 0.0)

    def adjoint(self, add, model, data):
        m = model.getNdArray()
        out = O.born_adjoint(O.Oracle("f"), self.case, data.getNdArray(), self.sig)
        m[...] = out + (m if add else 0.0)


def _run_script(name, argv):
    old = sys.argv
    sys.argv = [name] + argv
    try:
        runpy.run_path(os.path.join(SCRIPTS, name), run_name="__main__")
    finally:
        sys.argv = old


@pytest.mark.skipif(not os.path.isfile(os.path.join(SCRIPTS, "nonlinearPythonElasticFloatMain.py")),
                    reason="reference tree not present")
def test_reference_scripts_run_unchanged(tmp_path, monkeypatch, capsys):
    _, _, NL, BORN = _modules()
    monkeypatch.setattr(NL, "nonlinearPropElasticShotsGpu", _OracleNl)
    monkeypatch.setattr(BORN, "BornElasticShotsGpu", _OracleBorn)
    p, true_el, smooth_el, c_true, c_smooth, sig, dm = _write_inputs(tmp_path)
    orc = O.Oracle("f")
    f = lambda n: str(tmp_path / n)
    common = ["par=" + f("case.p"), "elasticParam=" + f("vpvsrho.H")]

    _run_script("nonlinearPythonElasticFloatMain.py", common + ["model=" + f("wavelet.H"), "data=" + f("d_nl.H")])
    d_nl = sepio.readSep(f("d_nl.H")).getNdArray()
    want = O.nl_forward(orc, c_true, sig[None])
    assert d_nl.shape == (NEXP, 5, 201, NTS)
    np.testing.assert_allclose(d_nl, want, rtol=0, atol=1e-6 * np.abs(want).max())

    _run_script("nonlinearPythonElasticFloatMain.py",
                common + ["adj=1", "model=" + f("src_adj.H"), "data=" + f("d_nl.H")])
    m_adj = sepio.readSep(f("src_adj.H"), ndims=4).getNdArray()
    want = O.nl_adjoint(orc, c_true, d_nl)
    assert O.rel_l2(m_adj.reshape(want.shape), want) < 1e-6

    born_args = ["sources=" + f("sources.H")]
    _run_script("BornPythonElasticFloatMain.py", common + born_args + ["model=" + f("dmodel.H"), "data=" + f("d_b.H")])
    d_b = sepio.readSep(f("d_b.H"), ndims=4).getNdArray()
    want = O.born_forward(orc, c_true, dm, [sig])
    assert O.rel_l2(d_b, want) < 1e-6 and np.abs(want).max() > 0

    _run_script("BornPythonElasticFloatMain.py",
                common + born_args + ["adj=1", "model=" + f("g_b.H"), "data=" + f("d_b.H")])
    g_b = sepio.readSep(f("g_b.H")).getNdArray()
    want = O.born_adjoint(orc, c_true, d_b, [sig])
    assert O.rel_l2(g_b, want) < 1e-6
    out = capsys.readouterr().out
    assert out.count("All done") == 4


@pytest.mark.gpu
def test_dropin_script_flow_on_the_engine_matches_oracle(tmp_path):
    """The scripts' sequence (set-up function, operator wrapper, forward or
    adjoint, writeVec) through the drop-in modules on the GPU engine."""
    P, G, _, _ = _modules()
    p, true_el, smooth_el, c_true, c_smooth, sig, dm = _write_inputs(tmp_path)
    orc = O.Oracle("f")
    f = lambda n: str(tmp_path / n)
    argv = ["prog", "par=" + f("case.p"), "elasticParam=" + f("vpvsrho.H")]

    # nonlinearPythonElasticFloatMain.py, forward then adjoint
    (model, data, elastic, par, sC, sX, sZ, sXZ, rC, rX, rZ, rXZ, modelLocal) = P.nonlinearOpInitFloat(argv)
    op = P.nonlinearPropElasticShotsGpu(model, data, elastic, par, sC, sX, sZ, sXZ, rC, rX, rZ, rXZ)
    wav = G.defaultIO.getVector(f("wavelet.H"))
    modelLocal.getNdArray()[0, :, 0, :] = wav.getNdArray()
    op.forward(False, modelLocal, data)
    data.writeVec(f("d_nl.H"))
    d_nl = sepio.readSep(f("d_nl.H")).getNdArray()
    want = O.nl_forward(orc, c_true, sig[None])
    assert O.rel_l2(d_nl, want) < TOL32
    dd = G.defaultIO.getVector(f("d_nl.H"), ndims=4)
    op.adjoint(False, modelLocal, dd)
    want = O.nl_adjoint(orc, c_true, d_nl)
    assert O.rel_l2(modelLocal.getNdArray(), want) < TOL32

    # BornPythonElasticFloatMain.py, forward then adjoint
    (bm, bd, bel, bpar, signals, sC, sX, sZ, sXZ, rC, rX, rZ, rXZ, bmLocal) = \
        P.BornOpInitFloat(argv + ["sources=" + f("sources.H")])
    bop = P.BornElasticShotsGpu(bm, bd, bel, bpar, signals, sC, sX, sZ, sXZ, rC, rX, rZ, rXZ)
    dmv = G.defaultIO.getVector(f("dmodel.H"))
    bop.forward(False, dmv, bd)
    want = O.born_forward(orc, c_true, dm, [sig])
    assert O.rel_l2(bd.getNdArray(), want) < TOL32
    bop.adjoint(False, bmLocal, bd)
    want = O.born_adjoint(orc, c_true, bd.getNdArray(), [sig])
    assert O.rel_l2(bmLocal.getNdArray(), want) < TOL32
    # the pySolver dot test of the wrapper (FP64 sums) passes too
    bop.dotTest(False, 1e-4)
