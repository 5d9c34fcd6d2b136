"""FWI host pieces on CPU: data-component sampling, parameter conversion and
its Jacobian, and the L-BFGS driver on a problem with a known minimiser."""
import numpy as np
import pytest

from elastic_isotropic_operators_b200 import fwi


def test_data_components_forward_adjoint():
    rng = np.random.default_rng(0)
    S = fwi.ElasticDatComp("p,vz,sxz")
    x = rng.standard_normal((2, 5, 7, 11)).astype(np.float32)
    y = rng.standard_normal(S.range_shape(x.shape)).astype(np.float32)
    Sx = np.zeros_like(y); S.forward(False, x, Sx)
    assert np.allclose(Sx[:, 0], 0.5 * (x[:, 2] + x[:, 3])) and np.array_equal(Sx[:, 1], x[:, 1])
    Sty = np.zeros_like(x); S.adjoint(False, Sty, y)
    assert abs(fwi.dot64(Sx, y) - fwi.dot64(x, Sty)) < 1e-6 * abs(fwi.dot64(Sx, y))
    with pytest.raises(ValueError):
        fwi.ElasticDatComp("vx,vx")
    with pytest.raises(ValueError):
        fwi.ElasticDatComp("vx,q")


@pytest.mark.parametrize("conv", [1, 2])
def test_conversion_jacobian(conv):
    rng = np.random.default_rng(1)
    scale = (1.0, 1.0, 1.0) if conv == 1 else (1e-3, 1e-3, 1e-3)
    bg = np.stack([rng.uniform(2000, 3000, (4, 6)) * scale[0], rng.uniform(900, 1300, (4, 6)) * scale[1],
                   rng.uniform(1800, 2400, (4, 6)) * scale[2]]).astype(np.float64)
    C = fwi.ElasticConv(conv)
    J = fwi.ElasticConvJab(bg.astype(np.float32), conv)
    dm = rng.standard_normal(bg.shape) * bg * 1e-3
    # directional derivative by central differences (FP64 inputs)
    def f(m):
        out = np.zeros_like(m); C.forward(False, m, out); return out
    h = 1e-3
    fd = (f(bg + h * dm) - f(bg - h * dm)) / (2 * h)
    Jdm = np.zeros(bg.shape, np.float32); J.forward(False, dm.astype(np.float32), Jdm)
    if conv == 2:
        # like the reference's setBackground, a km/s, g/cm3 background is scaled by 1e3
        # and the conversion-1 formulas apply to it
        Jdm_ref = np.zeros_like(Jdm)
        fwi.ElasticConvJab((bg * 1e3).astype(np.float32), 1).forward(False, dm.astype(np.float32), Jdm_ref)
        assert np.allclose(Jdm, Jdm_ref, rtol=1e-5)
    else:
        assert np.max(np.abs(Jdm - fd)) <= 1e-4 * np.max(np.abs(fd))
    y = rng.standard_normal(bg.shape).astype(np.float32)
    Jty = np.zeros_like(y); J.adjoint(False, Jty, y)
    assert abs(fwi.dot64(Jdm, y) - fwi.dot64(dm.astype(np.float32), Jty)) < 1e-5 * abs(fwi.dot64(Jdm, y))
    # round trip VpVsRho -> RhoLameMu -> VpVsRho (SI units)
    if conv == 1:
        back = np.zeros_like(bg); fwi.ElasticConv(-1).forward(False, f(bg), back)
        assert np.allclose(back, bg, rtol=1e-10)


class _Quadratic:
    """0.5 (m - m*)^T A (m - m*) with a diagonal, badly scaled A."""

    def __init__(self, n=20, seed=3):
        rng = np.random.default_rng(seed)
        self.a = np.logspace(0, 2, n)
        self.ms = rng.standard_normal(n)
        self.nfev = 0

    def value(self, m):
        r = m.astype(np.float64) - self.ms
        return 0.5 * float(np.sum(self.a * r * r))

    def value_and_gradient(self, m):
        r = m.astype(np.float64) - self.ms
        return 0.5 * float(np.sum(self.a * r * r)), (self.a * r).astype(np.float32)


def test_lbfgs_converges_and_respects_bounds():
    q = _Quadratic()
    m0 = np.full(20, 2.0, np.float32)
    m, hist = fwi.lbfgs(q, m0, niter=60, memory=10, init_step=0.5)
    assert all(b <= a for a, b in zip(hist, hist[1:]))
    assert hist[-1] < 1e-6 * hist[0]
    assert np.max(np.abs(m - q.ms)) < 1e-2
    lo = np.full(20, 0.0, np.float32)
    mb, hb = fwi.lbfgs(q, m0, niter=60, memory=10, minBound=lo, init_step=0.5)
    assert mb.min() >= 0.0
    want = np.maximum(q.ms, 0.0)
    assert np.max(np.abs(mb - want)) < 5e-2


class _SpreadQuadratic:
    """phi(m) = 0.5 (m - m*)^T A (m - m*) with a diagonal A of widely spread scales."""

    def __init__(self, n=60, seed=3):
        rng = np.random.default_rng(seed)
        self.a = np.exp(rng.uniform(-3, 3, n))
        self.mstar = rng.standard_normal(n)

    def value(self, m):
        d = np.asarray(m, np.float64) - self.mstar
        return 0.5 * float(d @ (self.a * d))

    def value_and_gradient(self, m):
        d = np.asarray(m, np.float64) - self.mstar
        return 0.5 * float(d @ (self.a * d)), (self.a * d).astype(np.float32)


def test_lbfgs_takes_good_learned_steps_and_rejects_bad_ones():
    q = _SpreadQuadratic()
    m0 = np.zeros(60, np.float32) + 0.5
    _, plain = fwi.lbfgs(q, m0, niter=6)
    # an (approximate) inverse Hessian: accepted, and it converges much faster
    good = {}
    _, learned = fwi.lbfgs(q, m0, niter=6, precond=lambda m, g: -g / (q.a * (1 + 0.05 * np.cos(np.arange(60)))),
                           stats=good)
    assert good["learned"] >= 1 and learned[2] < 1e-3 * plain[2]
    # a direction that increases the misfit is rejected; the plain steps still converge
    bad = {}
    _, fallback = fwi.lbfgs(q, m0, niter=6, precond=lambda m, g: g.astype(np.float64), stats=bad)
    assert bad["learned"] == 0 and bad["rejected"] >= 6
    assert fallback[-1] <= plain[-1] * 1.0001


def test_multiscale_runs_each_band_from_the_previous_model():
    seen = []

    class Band:
        def __init__(self, target):
            self.t = np.asarray(target, np.float64)

        def value(self, m):
            return 0.5 * float(np.sum((np.asarray(m, np.float64) - self.t) ** 2))

        def value_and_gradient(self, m):
            d = np.asarray(m, np.float64) - self.t
            return 0.5 * float(d @ d), d.astype(np.float32)

    targets = {(1, 2, 3, 4): np.full(8, 1.0), (1, 2, 6, 7): np.full(8, 2.0)}

    def for_band(band):
        seen.append(band)
        return Band(targets[band])

    starts, iters = [], []
    m, hists = fwi.multiscale(for_band, np.full(8, 0.5, np.float32), list(targets), niter=20, init_step=0.5,
                              callback=lambda k, band, mk, h: starts.append(mk.copy()),
                              iter_callback=lambda k, it, mk, f, g: iters.append((k, it, f)))
    assert seen == list(targets) and len(hists) == 2
    # the per-iteration hook sees every iteration of every band, tagged with the band, misfits as recorded
    for k in (0, 1):
        fk = [f for kk, it, f in iters if kk == k]
        assert [it for kk, it, f in iters if kk == k] == list(range(len(fk)))
        assert np.allclose(fk, hists[k][1:len(fk) + 1])
    assert np.allclose(starts[0], 1.0, atol=1e-3) and np.allclose(m, 2.0, atol=1e-3)
    # the second band started where the first ended: its first misfit is that of m = 1
    assert abs(hists[1][0] - 0.5 * 8 * 1.0) < 1e-2


def test_band_objective_filters_sources_and_data_for_both_operators():
    from elastic_isotropic_operators_b200 import wavelet

    class NL:
        sources = None

    class Born:
        fd = type("fd", (), {"surfaceCondition": 0})()
        sigs = None

        def setSourceSignals(self, s):
            self.sigs = [np.array(x) for x in s]

        def fwiGradient(self, *a):       # makes FwiObjective consider the fused path
            raise AssertionError("not called here")

    rng = np.random.default_rng(0)
    dts, nts = 1e-3, 256
    src = rng.standard_normal((2, 5, 1, nts)).astype(np.float32)
    d_obs = rng.standard_normal((2, 5, 3, nts)).astype(np.float32)
    nl, born = NL(), Born()
    nl.sources = src.copy()
    band = (2.0, 4.0, 20.0, 25.0)
    obj = fwi.band_objective(nl, born, d_obs, src, dts, band)
    want_src = wavelet.band_limit(src, dts, *band)
    assert np.allclose(nl.sources, want_src, atol=1e-6)
    assert len(born.sigs) == 2 and np.allclose(born.sigs[1], want_src[1], atol=1e-6)
    assert np.allclose(obj.d_obs, wavelet.band_limit(d_obs, dts, *band), atol=1e-6)
    # the band removes energy above 25 Hz
    spec = np.abs(np.fft.rfft(obj.d_obs, axis=-1))
    f = np.fft.rfftfreq(nts, dts)
    assert spec[..., f > 26].max() < 1e-4 * spec.max()
    assert obj.fused


def test_band_objective_never_filters_twice():
    """A band loop that passes ``nl.sources`` (or None) each time filters the
    broadband traces the operator was built with, not the previous band's."""
    from elastic_isotropic_operators_b200 import wavelet

    class NL:
        sources = None

    class Born:
        fd = type("fd", (), {"surfaceCondition": 0})()

        def setSourceSignals(self, s):
            self.sigs = [np.array(x) for x in s]

        def fwiGradient(self, *a):
            raise AssertionError("not called here")

    rng = np.random.default_rng(1)
    dts, nts = 1e-3, 256
    broadband = rng.standard_normal((1, 5, 1, nts)).astype(np.float32)
    d_obs = rng.standard_normal((1, 5, 3, nts)).astype(np.float32)
    nl, born = NL(), Born()
    nl.sources = broadband.copy()
    b1, b2 = (2.0, 4.0, 10.0, 14.0), (2.0, 4.0, 30.0, 36.0)
    fwi.band_objective(nl, born, d_obs, nl.sources, dts, b1)
    fwi.band_objective(nl, born, d_obs, nl.sources, dts, b2)
    assert np.allclose(nl.sources, wavelet.band_limit(broadband, dts, *b2), atol=1e-6)
    fwi.band_objective(nl, born, d_obs, None, dts, b1)
    assert np.allclose(nl.sources, wavelet.band_limit(broadband, dts, *b1), atol=1e-6)
    assert np.array_equal(nl._broadband_sources, broadband)
