"""Wavelets and band limitation for multiscale FWI (waveletFloatMain.py
restated): the band-limited wavelet against a loop-by-loop transcription of the
reference's construction (odd and even nts, with delay), its spectrum against
the trapezoid, the Ricker formula, the zero-phase band filter on traces."""
import numpy as np
import pytest

from elastic_isotropic_operators_b200 import wavelet as W


def _loop_wavelet(nts, dts, f1, f2, f3, f4, delay):
    """PF/waveletFloatMain.py:20-84, one frequency at a time."""
    odd = nts % 2 != 0
    n = nts + 1 if odd else nts
    spec = np.zeros(n, dtype=np.complex64)
    df = 1.0 / (n * dts)
    for i in range(n // 2):
        f = i * df
        if f < f1:
            spec[i] = 0
        elif f1 <= f < f2:
            spec[i] = np.cos(np.pi / 2.0 * (f2 - f) / (f2 - f1)) * np.cos(np.pi / 2.0 * (f2 - f) / (f2 - f1))
            spec[i] = spec[i] * np.exp(-1j * 2.0 * np.pi * f * delay)
        elif f2 <= f < f3:
            spec[i] = 1.0
            spec[i] = spec[i] * np.exp(-1j * 2.0 * np.pi * f * delay)
        elif f3 <= f < f4:
            spec[i] = np.cos(np.pi / 2.0 * (f - f3) / (f4 - f3)) * np.cos(np.pi / 2.0 * (f - f3) / (f4 - f3))
            spec[i] = spec[i] * np.exp(-1j * 2.0 * np.pi * f * delay)
        else:
            spec[i] = 0
    spec[n // 2 + 1:] = np.flip(spec[1:n // 2].conj(), axis=0)
    out = np.zeros(nts, np.float32)
    out[:] = np.fft.ifft(spec[:-1]).real if odd else np.fft.ifft(spec).real
    return out


@pytest.mark.parametrize("nts,delay", [(2000, 0.0), (1001, 0.25), (4000, 0.1)])
def test_band_wavelet_matches_loop_construction(nts, delay):
    args = (nts, 1e-3, 3.0, 5.0, 8.0, 10.0)
    got = W.band_wavelet(*args, timeDelay=delay)
    want = _loop_wavelet(*args, delay)
    np.testing.assert_allclose(got, want, rtol=0, atol=1e-6 * np.abs(want).max())


def test_band_wavelet_spectrum_is_the_trapezoid():
    nts, dts = 2048, 1e-3
    w = W.band_wavelet(nts, dts, 3.0, 5.0, 8.0, 10.0)
    f = np.fft.fftfreq(nts, dts)[: nts // 2]
    amp = np.abs(np.fft.fft(w.astype(np.float64)))[: nts // 2]
    np.testing.assert_allclose(amp, W.trapezoid(f, 3.0, 5.0, 8.0, 10.0), atol=1e-5)


def test_ricker():
    w = W.ricker_wavelet(500, 1e-3, 12.0, 0.1)
    t = np.arange(500) * 1e-3 - 0.1
    a = (np.pi * 12.0) ** 2
    np.testing.assert_allclose(w, (1 - 2 * a * t * t) * np.exp(-a * t * t), atol=1e-6)
    assert np.argmax(w) == 100


def test_band_limit_zero_phase_filter():
    rng = np.random.default_rng(3)
    x = rng.standard_normal((3, 4, 1024)).astype(np.float32)
    y = W.band_limit(x, 1e-3, 3.0, 5.0, 8.0, 10.0)
    assert y.dtype == np.float32 and y.shape == x.shape
    fx, fy = np.fft.rfft(x.astype(np.float64)), np.fft.rfft(y.astype(np.float64))
    f = np.fft.rfftfreq(1024, 1e-3)
    amp = W.trapezoid(f, 3.0, 5.0, 8.0, 10.0)
    np.testing.assert_allclose(np.abs(fy), np.abs(fx) * amp, atol=1e-3)
    flat = (f >= 5.0) & (f < 8.0)
    np.testing.assert_allclose(fy[..., flat], fx[..., flat], rtol=1e-5, atol=1e-4)   # no phase change


def test_corner_checks_and_bands():
    with pytest.raises(ValueError):
        W.band_wavelet(100, 1e-3, 5.0, 3.0, 8.0, 10.0)
    with pytest.raises(ValueError):
        W.band_wavelet(100, 1e-2, 3.0, 5.0, 8.0, 60.0)   # above Nyquist
    bands = W.multiscale_bands(3.0, 10.0, 4)
    assert len(bands) == 4 and bands[-1][2] == 10.0
    assert all(b[0] < b[1] <= b[2] < b[3] for b in bands)
    assert all(bands[i][2] < bands[i + 1][2] for i in range(3))
