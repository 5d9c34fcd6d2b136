"""CPU tests of the oracle itself (no GPU): closed-form constants, exact
adjointness of every restated operator in FP64 (the reference's own test
strategy: operator.h dotTest), and FP32-vs-FP64 agreement."""
import math

import numpy as np
import pytest

from oracle import oracle as O


def test_constants_closed_form():
    orc = O.Oracle("d")
    nts, dts, S, minPad = 100, 1e-3, 2, 12
    zc, xc, filt, damp = orc.consts(72, 104, 10.0, 12.5, nts, dts, S, minPad, 0.99)
    c = np.array([1.196289062541883, -0.079752604188901, 0.009570312506634, -6.975446437140719e-04])
    np.testing.assert_allclose(zc, c / 10.0, rtol=1e-15)
    np.testing.assert_allclose(xc, c / 12.5, rtol=1e-15)
    ntw = (nts - 1) * S + 1
    sc = 1.0 / math.sqrt(ntw / nts)
    h = S + 1
    want = [(1 - i / S) * sc for i in range(h)] + [(i / S) * sc for i in range(h)]
    np.testing.assert_allclose(filt, want, rtol=1e-14)
    dwant = [0.99 + 0.01 * math.cos(math.pi * (minPad - d) / minPad) for d in range(minPad)]
    np.testing.assert_allclose(damp, dwant, rtol=1e-7)   # alphaCos is float-rounded like getFloat
    assert np.all(np.diff(damp) >= 0)


def test_stagger_adjoint():
    orc = O.Oracle("d")
    rng = np.random.default_rng(0)
    for ax in (0, 1):
        m = rng.standard_normal((23, 17))
        d = rng.standard_normal((23, 17))
        Sm = np.zeros_like(d)
        orc.stagger(ax, 0, 0, m.copy(), Sm)
        Std = np.zeros_like(m)
        orc.stagger(ax, 1, 0, Std, d.copy())
        assert abs(np.vdot(Sm, d) - np.vdot(m, Std)) < 1e-12 * abs(np.vdot(Sm, d))


def test_medium_closed_form(small_case):
    w = small_case
    orc = O.Oracle("d")
    ep = w.elastic.getNdArray().astype(np.float64)
    rx, rz, l2m, lam, mu = orc.medium(ep, w.dts, 2 * w.sub)
    dtw = float(np.float32(w.dts)) / (2 * w.sub)
    rho = ep[0]
    np.testing.assert_allclose(rx[1:-1], 2 * dtw / (0.5 * (rho[1:-1] + rho[:-2])), rtol=1e-14)
    np.testing.assert_allclose(rz[:, 1:-1], 2 * dtw / (0.5 * (rho[:, 1:-1] + rho[:, :-2])), rtol=1e-14)
    np.testing.assert_allclose(l2m, 2 * dtw * (ep[1] + 2 * ep[2]), rtol=1e-14)
    np.testing.assert_allclose(lam, 2 * dtw * ep[1], rtol=1e-14)
    m = ep[2]
    mxz = 0.25 * (m[1:-1, 1:-1] + m[:-2, 1:-1] + m[1:-1, :-2] + m[:-2, :-2])
    np.testing.assert_allclose(mu[1:-1, 1:-1], 2 * dtw * mxz, rtol=1e-13)


def test_time_interp_adjoint_and_exact_on_lines():
    orc = O.Oracle("d")
    nts, S = 40, 4
    ntw = (nts - 1) * S + 1
    rng = np.random.default_rng(1)
    m = rng.standard_normal((3, nts))
    f = rng.standard_normal((3, ntw))
    Fm = np.zeros((3, ntw))
    orc.tinterp(0, 0, nts, 2e-3, 0.0, S, m.copy(), Fm)
    Ftf = np.zeros((3, nts))
    orc.tinterp(1, 0, nts, 2e-3, 0.0, S, Ftf, f.copy())
    assert abs(np.vdot(Fm, f) - np.vdot(m, Ftf)) < 1e-12 * abs(np.vdot(Fm, f))
    lin = np.tile(np.arange(nts, dtype=np.float64), (1, 1))
    out = np.zeros((1, ntw))
    orc.tinterp(0, 0, nts, 2e-3, 0.0, S, lin, out)
    scale = 1.0 / math.sqrt(float(np.float32(ntw) / np.float32(nts)))
    np.testing.assert_allclose(out[0] / scale, np.arange(ntw) / S, atol=2e-5)


@pytest.mark.parametrize("method,nfilt", [("linear", 1), ("sinc", 1), ("sinc", 2), ("gauss", 2)])
def test_space_interp_weights(method, nfilt):
    orc = O.Oracle("d")
    rng = np.random.default_rng(2)
    zc = rng.uniform(100, 400, 9)
    xc = rng.uniform(100, 600, 9)
    s = orc.sinterp(zc, xc, 60, 0.0, 10.0, 80, -5.0, 10.0, method, nfilt)
    w = s["w"].reshape(9, -1)
    np.testing.assert_allclose(w.sum(axis=1), 1.0, rtol=1e-12)
    assert len(set(s["uniq"].tolist())) == len(s["uniq"])
    # forward / adjoint are transposes
    reg = rng.standard_normal((len(s["uniq"]), 7))
    irr = rng.standard_normal((9, 7))
    Fr = np.zeros_like(irr)
    orc.sinterp_apply(s, 0, 0, reg.copy(), Fr)
    Fti = np.zeros_like(reg)
    orc.sinterp_apply(s, 1, 0, Fti, irr.copy())
    assert abs(np.vdot(Fr, irr) - np.vdot(reg, Fti)) < 1e-12 * abs(np.vdot(Fr, irr))


def test_space_interp_linear_on_grid_point():
    orc = O.Oracle("f")
    s = orc.sinterp(np.float32([50.0]), np.float32([80.0]), 30, 0.0, 10.0, 30, 0.0, 10.0)
    np.testing.assert_array_equal(s["uniq"], [8 * 30 + 5, 8 * 30 + 6, 9 * 30 + 5, 9 * 30 + 6])
    np.testing.assert_array_equal(s["w"], [1.0, 0.0, 0.0, 0.0])


def test_space_interp_bounds():
    orc = O.Oracle("f")
    with pytest.raises(ValueError):
        orc.sinterp(np.float32([5.0]), np.float32([80.0]), 30, 0.0, 10.0, 30, 0.0, 10.0)


def _dot(a, b):
    return float(np.dot(np.ravel(a).astype(np.float64), np.ravel(b).astype(np.float64)))


def test_nl_dot_product_fp64(small_case):
    w = small_case
    orc = O.Oracle("d")
    c = O.Case.from_workload(w)
    rng = np.random.default_rng(3)
    m = rng.standard_normal((1, 5, 1, w.nts))
    d = rng.standard_normal((w.nExp, 5, w.rec_z.size, w.nts))
    a = _dot(O.nl_forward(orc, c, m), d)
    b = _dot(m, O.nl_adjoint(orc, c, d))
    assert abs(a - b) / abs(b) < 1e-11


def test_born_dot_product_fp64(small_case):
    w = small_case
    orc = O.Oracle("d")
    c = O.Case.from_workload(w)
    rng = np.random.default_rng(4)
    m = rng.standard_normal((3, w.nx, w.nz))
    d = rng.standard_normal((w.nExp, 5, w.rec_z.size, w.nts))
    sig = [w.source_signal()]
    a = _dot(O.born_forward(orc, c, m, sig), d)
    b = _dot(m, O.born_adjoint(orc, c, d, sig))
    assert abs(a - b) / abs(b) < 1e-11


def test_fp32_vs_fp64(small_case):
    w = small_case
    c = O.Case.from_workload(w)
    m = w.source_signal()[None]
    d32 = O.nl_forward(O.Oracle("f"), c, m)
    d64 = O.nl_forward(O.Oracle("d"), c, m)
    assert O.rel_l2(d32, d64) < 1e-5
    dm = w.extra["dmodel"]
    b32 = O.born_forward(O.Oracle("f"), c, dm, [w.source_signal()])
    b64 = O.born_forward(O.Oracle("d"), c, dm, [w.source_signal()])
    assert O.rel_l2(b32, b64) < 1e-4


def test_born_is_derivative_of_nonlinear(small_case):
    """Taylor test: [F(m + h dm) - F(m - h dm)] / 2h vs Born(dm) (FP64).

    The reference's Born operator builds its secondary sources from the
    coarse-time history of Vx/Vz (time derivative (W[its-1] - W[its+1]) / 2dts)
    and interpolates them to the fine steps, so it is the derivative of the
    nonlinear operator only up to that time discretisation: the mismatch
    stays near 1% for every h instead of vanishing.  A wrong sign or scale of
    any of the five secondary sources would give an O(1) mismatch."""
    w = small_case
    orc = O.Oracle("d")
    ep = w.elastic.getNdArray().astype(np.float64)
    dm = w.extra["dmodel"].astype(np.float64)
    src = w.source_signal()[None]
    c = O.Case.from_workload(w)
    born = O.born_forward(orc, c, dm, [w.source_signal()])
    errs = []
    for h in (1e-2, 5e-3):
        cp = O.Case(ep + h * dm, w.par.as_dict(), w.oz, w.ox, c.src, c.rec)
        cm = O.Case(ep - h * dm, w.par.as_dict(), w.oz, w.ox, c.src, c.rec)
        fd = (O.nl_forward(orc, cp, src) - O.nl_forward(orc, cm, src)) / (2 * h)
        errs.append(O.rel_l2(born, fd))
    assert max(errs) < 3e-2
    assert abs(errs[0] - errs[1]) < 0.1 * errs[0]   # h-independent: no nonlinear residue left


@pytest.mark.parametrize("adj", [0, 1])
def test_saved_wavefield_equals_traces_at_the_devices(adj):
    """The saved wavefield (interpWavefield, K:1258-1291) and the recorded traces
    (K:7-60, 100-116) are the same coarse-time samples of the same level, so at
    the receiver cells (forward) or source cells (adjoint, before scaling) they
    agree exactly."""
    from elastic_isotropic_operators_b200 import synthetic
    from helpers import reg_inputs
    w = synthetic.small(nts=60)
    r = reg_inputs(w, "f", seed=3)
    orc, g = r["orc"], r["g"]
    W = np.zeros((g["nts"], 5, g["nx"], g["nz"]), np.float32)
    m = [x.copy() for x in r["model"]]
    d = [x.copy() for x in r["data"]]
    orc.nl_prop(adj, g, r["med"], m, d, r["sp"], r["rp"], W)
    traces, pos = (m, r["sp"]) if adj else (d, r["rp"])
    flat = W.reshape(g["nts"], 5, -1)
    for f in range(5):
        got = flat[:, f, pos[O.FIELD_GRID[f]]].T
        assert np.array_equal(got, traces[f]), f
    assert np.abs(W).max() > 0
    # nothing is written outside the updated interior
    assert not W[:, :, :4].any() and not W[:, :, -4:].any()
    assert not W[..., :4].any() and not W[..., -4:].any()


@pytest.mark.parametrize("alpha,tol", [(1.0, 1e-12), (0.99, 1e-6)])
def test_free_surface_forward_adjoint_dot_product(alpha, tol):
    """Free surface (surfaceCondition = 1): the oracle's adjoint step (masked
    products, transposed stencils, transpose of the top mirroring) against its
    forward step (top mirroring, masked update, reduced sigmaxx coefficient on
    the surface).  Without the taper (alphaCos = 1) the pair is adjoint to
    rounding; the taper brings the same small deviation as without the free
    surface (the damping is applied after the update in both directions)."""
    from elastic_isotropic_operators_b200 import synthetic
    from helpers import reg_inputs
    w = synthetic.small(nts=80, surface=1, alphaCos=alpha)
    r = reg_inputs(w, "d", seed=9)
    orc, g = r["orc"], r["g"]
    assert g["surface"] == 1
    m = [x.copy() for x in r["model"]]
    d = [x.copy() for x in r["data"]]
    fd = [np.zeros_like(x) for x in d]
    orc.nl_prop(0, g, r["med"], m, fd, r["sp"], r["rp"])
    am = [np.zeros_like(x) for x in m]
    orc.nl_prop(1, g, r["med"], am, d, r["sp"], r["rp"])
    lhs = sum(float(np.dot(a.ravel(), b.ravel())) for a, b in zip(fd, d))
    rhs = sum(float(np.dot(a.ravel(), b.ravel())) for a, b in zip(m, am))
    assert abs(lhs - rhs) <= tol * abs(lhs), (lhs, rhs, abs(lhs - rhs) / abs(lhs))
    # the surface changes the result
    g0 = dict(g, surface=0)
    fd0 = [np.zeros_like(x) for x in d]
    orc.nl_prop(0, g0, r["med"], m, fd0, r["sp"], r["rp"])
    assert sum(float(np.abs(a - b).max()) for a, b in zip(fd, fd0)) > 0
