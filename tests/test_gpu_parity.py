"""Parity of the sm_100a engine (through the C ABI) with the CPU oracle and with
the reference's own CUDA drivers (oracle/_ref), plus adjointness.

Tolerances (relative L2 over the whole output):
  FP32 engine vs FP32 oracle / reference float build   <= 1e-5
  FP32 engine vs FP64 oracle (elastic_iso_double)       <= 1e-4 (nonlinear), 1e-4 (Born)
  dot-product tests (FP64 reductions)                    <= 1e-5
  reference float build vs FP32 oracle                   <= 1e-5
  reference double build vs FP64 oracle                  <= 1e-10
"""
import numpy as np
import pytest

from elastic_isotropic_operators_b200 import prop, synthetic
from oracle import oracle as O

from helpers import Ctx, reg_inputs, rel

pytestmark = pytest.mark.gpu

TOL32 = 1e-5
TOL64 = 1e-4


@pytest.fixture(scope="module")
def w():
    return synthetic.small()


@pytest.fixture(scope="module")
def ctx(w):
    c = Ctx(w)
    yield c
    c.close()


def _copy(xs):
    return [x.copy() for x in xs]


@pytest.mark.parametrize("adj", [0, 1])
def test_nl_reg_vs_oracle(w, ctx, adj):
    for prec, tol in (("f", TOL32), ("d", TOL64)):
        r = reg_inputs(w, prec)
        orc = r["orc"]
        m, d = _copy(r["model"]), _copy(r["data"])
        orc.nl_prop(adj, r["g"], r["med"], m, d, r["sp"], r["rp"])
        pm, pd = ctx.nl(adj, r["model"], r["data"], r["sp"], r["rp"])
        got, want = (pm, m) if adj else (pd, d)
        assert rel(got, want) < tol, (prec, rel(got, want))


@pytest.mark.parametrize("adj", [0, 1])
def test_born_reg_vs_oracle(w, ctx, adj):
    for prec, tol in (("f", TOL32), ("d", TOL64)):
        r = reg_inputs(w, prec)
        orc = r["orc"]
        dm, d = _copy(r["dm"]), _copy(r["data"])
        orc.born_prop(adj, r["g"], r["med"], r["fine"], dm, d, r["sp"], r["rp"])
        pdm, pd = ctx.born(adj, r["fine"], r["dm"], r["data"], r["sp"], r["rp"])
        got, want = (pdm, dm) if adj else (pd, d)
        assert rel(got, want) < tol, (prec, rel(got, want))


def _ops(w, nModelExp=1, per_shot_rec=False, method="linear", nfilt=1):
    src, rec = w.geometry(method, nfilt)
    if per_shot_rec:
        rec = [g * w.nExp for g in rec]
    nl = prop.nonlinearPropElasticShotsGpu(w.elastic, w.par, *src, *rec)
    return nl, src, rec


def test_nl_operator_vs_oracle(w):
    nl, src, rec = _ops(w)
    c = O.Case.from_workload(w)
    model = nl.modelSpace()
    model.getNdArray()[...] = w.source_signal()[None]
    data = nl.dataSpace()
    nl.forward(False, model, data)
    want = O.nl_forward(O.Oracle("f"), c, model.getNdArray())
    assert O.rel_l2(data.getNdArray(), want) < TOL32
    want64 = O.nl_forward(O.Oracle("d"), c, model.getNdArray())
    assert O.rel_l2(data.getNdArray(), want64) < TOL64
    # add = True accumulates
    d0 = data.getNdArray().copy()
    nl.forward(True, model, data)
    assert O.rel_l2(data.getNdArray(), 2 * d0) < 1e-6
    # adjoint, constant source signal: shots are stacked
    rng = np.random.default_rng(8)
    dd = nl.dataSpace()
    dd.getNdArray()[...] = rng.standard_normal(dd.getNdArray().shape)
    m2 = nl.modelSpace()
    nl.adjoint(False, m2, dd)
    want = O.nl_adjoint(O.Oracle("f"), c, dd.getNdArray(), 1)
    assert O.rel_l2(m2.getNdArray(), want) < TOL32


def test_nl_operator_per_shot_signals_and_receivers(w):
    nl, src, rec = _ops(w, per_shot_rec=True)
    c = O.Case.from_workload(w)
    rng = np.random.default_rng(9)
    model = nl.modelSpace(nModelExp=w.nExp)
    model.getNdArray()[...] = rng.standard_normal(model.getNdArray().shape)
    data = nl.dataSpace()
    nl.forward(False, model, data)
    want = O.nl_forward(O.Oracle("f"), c, model.getNdArray())
    assert O.rel_l2(data.getNdArray(), want) < TOL32
    m2 = nl.modelSpace(nModelExp=w.nExp)
    nl.adjoint(False, m2, data)
    want = O.nl_adjoint(O.Oracle("f"), c, data.getNdArray(), w.nExp)
    assert O.rel_l2(m2.getNdArray(), want) < TOL32


def test_nl_operator_sinc_geometry(w):
    nl, src, rec = _ops(w, method="sinc", nfilt=1)
    c = O.Case.from_workload(w, "sinc", 1)
    model = nl.modelSpace()
    model.getNdArray()[...] = w.source_signal()[None]
    data = nl.dataSpace()
    nl.forward(False, model, data)
    assert O.rel_l2(data.getNdArray(), O.nl_forward(O.Oracle("f"), c, model.getNdArray())) < TOL32


def test_born_operator_vs_oracle(w):
    src, rec = w.geometry()
    sig = [w.source_signal()]
    born = prop.BornElasticShotsGpu(w.elastic, w.par, sig, *src, *rec)
    c = O.Case.from_workload(w)
    dm = born.modelSpace()
    dm.getNdArray()[...] = w.extra["dmodel"]
    data = born.dataSpace()
    born.forward(False, dm, data)
    assert O.rel_l2(data.getNdArray(), O.born_forward(O.Oracle("f"), c, dm.getNdArray(), sig)) < TOL32
    assert O.rel_l2(data.getNdArray(), O.born_forward(O.Oracle("d"), c, dm.getNdArray(), sig)) < TOL64
    g = born.modelSpace()
    born.adjoint(False, g, data)
    want = O.born_adjoint(O.Oracle("f"), c, data.getNdArray(), sig)
    assert O.rel_l2(g.getNdArray(), want) < TOL32
    want64 = O.born_adjoint(O.Oracle("d"), c, data.getNdArray(), sig)
    assert O.rel_l2(g.getNdArray(), want64) < TOL64


def test_prepare_shot_matches_oracle_host_prep(w):
    """Host preparation the single-shot device entry points are fed with:
    nonlinear spread + scaling of the source traces, Born fine-time sources and
    the staggered model perturbation; the oracle restates the same steps."""
    src, rec = w.geometry()
    sig = w.source_signal()
    orc = O.Oracle("f")
    c = O.Case.from_workload(w)
    g = c.grid()
    med = orc.medium(c.ep, g["dts"], g["S"])
    sg = O._grids(orc, c, *c.src[1])
    nl = prop.nonlinearPropElasticShotsGpu(w.elastic, w.par, *src, *rec)
    reg, sp, rp = nl.prepareShot(1, sig)
    want = []
    for f in range(5):
        G = sg[O.FIELD_GRID[f]]
        r = np.zeros((len(G["uniq"]), g["nts"]), np.float32)
        orc.sinterp_apply(G, 1, 0, r, np.ascontiguousarray(sig[f]))
        want.append(r)
    O._scale_sources(orc, g, med, sg, want)
    assert rel(reg, want) < 1e-6
    for k in range(4):
        assert np.array_equal(sp[k], sg[k]["uniq"])
    born = prop.BornElasticShotsGpu(w.elastic, w.par, [sig], *src, *rec)
    fine, sp2, _ = born.prepareShot(1)
    want_fine = O.born_sources(orc, c, g, med, sg, sig.reshape(5, 1, g["nts"]))
    assert rel(fine, want_fine) < 1e-6
    dm = born.prepareModel(w.extra["dmodel"])
    assert rel(dm, O.born_model_slice(orc, g, med, w.extra["dmodel"])) < 1e-6


def test_dot_products(w):
    nl, src, rec = _ops(w)
    assert nl.dotTest(False, 1e-5), nl.lastDotTest
    born = prop.BornElasticShotsGpu(w.elastic, w.par, [w.source_signal()], *src, *rec)
    assert born.dotTest(False, 1e-5), born.lastDotTest


def test_set_background(w):
    nl, src, rec = _ops(w)
    ep2 = w.elastic.clone()
    ep2.getNdArray()[0] *= 1.1
    nl.setBackground(ep2)
    model = nl.modelSpace()
    model.getNdArray()[...] = w.source_signal()[None]
    data = nl.dataSpace()
    nl.forward(False, model, data)
    c = O.Case(ep2.getNdArray(), w.par.as_dict(), w.oz, w.ox, O.Case.from_workload(w).src, (w.rec_z, w.rec_x))
    assert O.rel_l2(data.getNdArray(), O.nl_forward(O.Oracle("f"), c, model.getNdArray())) < TOL32
    bad = w.elastic.clone()
    bad.getNdArray()[1] *= 100.0     # Courant violation
    with pytest.raises(prop.EioError):
        nl.setBackground(bad)


def test_out_of_interior_point_rejected(w, ctx):
    r = reg_inputs(w, "f")
    sp = [p.copy() for p in r["sp"]]
    sp[0][0] = 1     # inside the FAT frame
    with pytest.raises(prop.EioError):
        ctx.nl(0, r["model"], r["data"], sp, r["rp"])


# ------------------------------------------------------------------ every step-kernel variant
KERNELS = [(0, 64, 16, 0), (2, 64, 16, 0), (3, 64, 16, 0), (4, 64, 16, 0), (5, 64, 16, 0), (1, 64, 8, 4), (1, 64, 8, 5), (1, 64, 16, 2), (1, 64, 16, 1), (1, 128, 8, 3)]


@pytest.mark.parametrize("cfg", KERNELS, ids=lambda c: "k%d_tz%d_cw%d_cpr%d" % c)
def test_kernel_variants_vs_oracle(w, cfg):
    c = Ctx(w)
    try:
        c.set_kernel(*cfg)
        r = reg_inputs(w, "f", seed=5)
        orc = r["orc"]
        for adj in (0, 1):
            m, d = _copy(r["model"]), _copy(r["data"])
            orc.nl_prop(adj, r["g"], r["med"], m, d, r["sp"], r["rp"])
            pm, pd = c.nl(adj, r["model"], r["data"], r["sp"], r["rp"])
            assert rel(pm if adj else pd, m if adj else d) < TOL32, ("nl", adj)
            dm, d = _copy(r["dm"]), _copy(r["data"])
            orc.born_prop(adj, r["g"], r["med"], r["fine"], dm, d, r["sp"], r["rp"])
            pdm, pd = c.born(adj, r["fine"], r["dm"], r["data"], r["sp"], r["rp"])
            assert rel(pdm if adj else pd, dm if adj else d) < TOL32, ("born", adj)
        assert c.get_kernel()[0] == cfg[0]
    finally:
        c.close()


def test_autotune_picks_a_valid_kernel(w):
    c = Ctx(w)
    try:
        kind, tz, cw, cpr = c.autotune()
        assert kind in (0, 1, 2, 3, 4, 5)
        if kind == 1:
            assert tz in (64, 128) and cw in (8, 16) and cpr >= 1
        with pytest.raises(prop.EioError):
            c.set_kernel(1, 96, 8, 4)
    finally:
        c.close()


# ------------------------------------------------------------------ reference's own CUDA build
ref_available = O.RefGpu.available("f") and O.RefGpu.available("d")


@pytest.mark.skipif(not ref_available, reason="oracle/_ref not built")
@pytest.mark.parametrize("kind", ["nl_fwd", "nl_adj", "born_fwd", "born_adj"])
def test_reference_gpu_pins_oracle_and_engine(w, ctx, kind):
    adj = int(kind.endswith("adj"))
    for prec, tol in (("f", TOL32), ("d", 1e-10)):
        r = reg_inputs(w, prec)
        orc, refg = r["orc"], O.RefGpu(prec)
        if kind.startswith("nl"):
            mo, do = _copy(r["model"]), _copy(r["data"])
            orc.nl_prop(adj, r["g"], r["med"], mo, do, r["sp"], r["rp"])
            mr, dr = _copy(r["model"]), _copy(r["data"])
            refg.nl_prop(adj, r["g"], r["med"], mr, dr, r["sp"], r["rp"])
            want, got_ref = (mo, mr) if adj else (do, dr)
            if prec == "f":
                pm, pd = ctx.nl(adj, r["model"], r["data"], r["sp"], r["rp"])
                assert rel(pm if adj else pd, got_ref) < TOL32
        else:
            dmo, do = _copy(r["dm"]), _copy(r["data"])
            orc.born_prop(adj, r["g"], r["med"], r["fine"], dmo, do, r["sp"], r["rp"])
            dmr, dr = _copy(r["dm"]), _copy(r["data"])
            refg.born_prop(adj, r["g"], r["med"], r["fine"], dmr, dr, r["sp"], r["rp"])
            want, got_ref = (dmo, dmr) if adj else (do, dr)
            if prec == "f":
                pdm, pd = ctx.born(adj, r["fine"], r["dm"], r["data"], r["sp"], r["rp"])
                assert rel(pdm if adj else pd, got_ref) < TOL32
        assert rel(got_ref, want) < tol, (prec, kind, rel(got_ref, want))


# ------------------------------------------------------------------ full-size properties
def test_full_size_nl_312x520_vs_oracle():
    """The nonlinear benchmark case at full size (312x520, 3998 fine steps)."""
    w = synthetic.nl_312x520()
    src, rec = w.geometry()
    nl = prop.nonlinearPropElasticShotsGpu(w.elastic, w.par, *src, *rec)
    model = nl.modelSpace()
    model.getNdArray()[...] = w.source_signal()[None]
    data = nl.dataSpace()
    nl.forward(False, model, data)
    want = O.nl_forward(O.Oracle("f"), O.Case.from_workload(w), model.getNdArray())
    assert O.rel_l2(data.getNdArray(), want) < TOL32
    assert np.abs(data.getNdArray()).max() > 0


def test_full_size_born_600x1800_dot_product():
    """Born adjointness on the 600x1800, nts=4000 benchmark grid (one shot)."""
    w = synthetic.born_600x1800(nshots=1)
    src, rec = w.geometry()
    born = prop.BornElasticShotsGpu(w.elastic, w.par, [w.source_signal()], *src, *rec)
    assert born.dotTest(False, 1e-5), born.lastDotTest


def _nl_born_vs_oracle(c, w, seed):
    r = reg_inputs(w, "f", seed=seed)
    orc = r["orc"]
    for adj in (0, 1):
        dm, d = _copy(r["dm"]), _copy(r["data"])
        orc.born_prop(adj, r["g"], r["med"], r["fine"], dm, d, r["sp"], r["rp"])
        pdm, pd = c.born(adj, r["fine"], r["dm"], r["data"], r["sp"], r["rp"])
        assert rel(pdm if adj else pd, dm if adj else d) < TOL32, ("born", adj)
        m, d = _copy(r["model"]), _copy(r["data"])
        orc.nl_prop(adj, r["g"], r["med"], m, d, r["sp"], r["rp"])
        pm, pd = c.nl(adj, r["model"], r["data"], r["sp"], r["rp"])
        assert rel(pm if adj else pd, m if adj else d) < TOL32, ("nl", adj)


@pytest.mark.parametrize("kind", [0, 1, 2, 3, 4, 5])
def test_ragged_tiles_vs_oracle(kind):
    """A grid whose interior (96 x 112) leaves a half-height last tile row, so the
    TMA boxes reach past the grid edge and read the zero fill."""
    w = synthetic.small(nz=104, nx=120, nts=80)
    c = Ctx(w)
    try:
        c.set_kernel(kind, 64, 16, 2)
        _nl_born_vs_oracle(c, w, 17)
    finally:
        c.close()


@pytest.mark.parametrize("kind", [None, 0, 2, 3, 4, 5])
def test_sub2_running_sum_path_vs_oracle(kind):
    """sub = 2 (four fine steps per coarse sample) keeps the running-sum history
    and adjoint accumulation; sub = 1 (every other test) takes the single-write path."""
    w2 = synthetic.small(nts=60, sub=2)
    c = Ctx(w2)
    try:
        if kind is not None:
            c.set_kernel(kind, 64, 16, 0)
        _nl_born_vs_oracle(c, w2, 13)
    finally:
        c.close()


# ------------------------------------------------------------------ wavefield output
def _wavefield_op(w, shot):
    from elastic_isotropic_operators_b200.sepvec import paramObj
    par = paramObj(w.par.as_dict())
    par.set("saveWavefield", "1")
    par.set("wavefieldShotNumber", str(shot))
    src, rec = w.geometry()
    return prop.nonlinearPropElasticShotsGpu(w.elastic, par, *src, *rec)


@pytest.mark.parametrize("adj", [0, 1])
def test_nl_wavefield_operator_vs_oracle(w, adj):
    """forwardWavefield / adjointWavefield keep the wavefield of shot
    wavefieldShotNumber; the adjoint one scaled like the adjoint sources."""
    nl = _wavefield_op(w, 1)
    c = O.Case.from_workload(w)
    orc = O.Oracle("f")
    rng = np.random.default_rng(8)
    model, data = nl.modelSpace(), nl.dataSpace()
    if not adj:
        model.getNdArray()[...] = w.source_signal()[None]
        nl.forwardWavefield(False, model, data)
        want, wantW = O.nl_forward(orc, c, model.getNdArray(), wshot=1)
        got = data.getNdArray()
    else:
        data.getNdArray()[...] = rng.standard_normal(data.getNdArray().shape).astype(np.float32)
        nl.adjointWavefield(False, model, data)
        want, wantW = O.nl_adjoint(orc, c, data.getNdArray(), wshot=1)
        got = model.getNdArray()
    W = nl.getWavefield().getNdArray()
    assert W.shape == (w.nts, 5, w.nx, w.nz)
    assert O.rel_l2(got, want) < TOL32
    assert O.rel_l2(W, wantW) < TOL32, O.rel_l2(W, wantW)
    assert np.abs(W).max() > 0


def test_nl_wavefield_off_keeps_no_wavefield(w):
    from elastic_isotropic_operators_b200.sepvec import paramObj
    src, rec = w.geometry()
    nl = prop.nonlinearPropElasticShotsGpu(w.elastic, paramObj(w.par.as_dict()), *src, *rec)
    model, data = nl.modelSpace(), nl.dataSpace()
    model.getNdArray()[...] = w.source_signal()[None]
    nl.forwardWavefield(False, model, data)
    assert nl.getWavefield().getNdArray().size == 1
    ref = nl.dataSpace()
    nl.forward(False, model, ref)
    assert np.array_equal(ref.getNdArray(), data.getNdArray())


@pytest.mark.skipif(not ref_available, reason="oracle/_ref not built")
@pytest.mark.parametrize("adj", [0, 1])
def test_reference_wavefield_pins_oracle(w, adj):
    """The reference's own wavefield drivers agree with the oracle on every cell
    they write; their kernel omits the FAT offset in z (K:1262), so the last four
    interior rows stay zero there."""
    for prec, tol in (("f", TOL32), ("d", 1e-10)):
        r = reg_inputs(w, prec, seed=21)
        g = r["g"]
        orc, ref = r["orc"], O.RefGpu(prec)
        Wo = np.zeros((g["nts"], 5, g["nx"], g["nz"]), orc.dt)
        Wr = np.zeros_like(Wo)
        mo, do_ = _copy(r["model"]), _copy(r["data"])
        mr, dr = _copy(r["model"]), _copy(r["data"])
        orc.nl_prop(adj, g, r["med"], mo, do_, r["sp"], r["rp"], Wo)
        ref.nl_prop(adj, g, r["med"], mr, dr, r["sp"], r["rp"], Wr)
        nz = g["nz"]
        assert not Wr[..., nz - 8:nz - 4].any()
        assert O.rel_l2(Wr[..., :nz - 8], Wo[..., :nz - 8]) < tol, (prec, adj)


def test_nonlinear_fwi_operator_sets_background_then_propagates(w):
    """nonlinearFwiPropElasticShotsGpu.forward(model) = setBackground(model) + forward(sources)."""
    src, rec = w.geometry()
    sig = w.source_signal()[None]
    fwi = prop.nonlinearFwiPropElasticShotsGpu(w.elastic, w.par, sig, *src, *rec)
    nl = prop.nonlinearPropElasticShotsGpu(w.elastic, w.par, *src, *rec)
    # bitwise comparison: both contexts on the same kernel (each would autotune on its own)
    from elastic_isotropic_operators_b200 import _lib
    for op in (fwi, nl):
        _lib.check(op._L.eio_ctx_set_kernel(op.ctx, 0, 64, 16, 0))
    model2 = w.elastic.clone()
    model2.getNdArray()[...] = w.elastic.getNdArray() * np.float32(1.02)
    d_fwi = fwi.dataSpace()
    fwi.forward(False, model2, d_fwi)
    nl.setBackground(model2)
    d_nl = nl.dataSpace()
    m = nl.modelSpace()
    m.getNdArray()[...] = sig
    nl.forward(False, m, d_nl)
    assert np.array_equal(d_fwi.getNdArray(), d_nl.getNdArray())
    with pytest.raises(NotImplementedError):
        fwi.adjoint(False, model2, d_fwi)
