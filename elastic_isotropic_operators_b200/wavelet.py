"""Source wavelets and band limitation for multiscale FWI.

The reference builds its source signals with ``waveletFloatMain.py``
(PF/waveletFloatMain.py:13-86 band-limited "ali" wavelet, :89-108 Ricker) and
runs its multiscale FWI by swapping in wavelets of growing bandwidth.  This
module restates both wavelets without genericIO and adds ``band_limit``, the
same trapezoid applied with zero phase to existing traces (observed data or a
wavelet), so that every band of a multiscale run sees consistent sources and
data.

Trapezoid (corner frequencies f1 < f2 <= f3 < f4): 0 below f1,
cos^2(pi/2 (f2 - f) / (f2 - f1)) on [f1, f2), 1 on [f2, f3),
cos^2(pi/2 (f - f3) / (f4 - f3)) on [f3, f4), 0 from f4 on.
"""
import numpy as np

__all__ = ["trapezoid", "band_wavelet", "ricker_wavelet", "band_limit", "multiscale_bands"]


def _check_corners(f1, f2, f3, f4, dts):
    if not (f1 < f2 <= f3 < f4):
        raise ValueError("corner frequencies must satisfy f1 < f2 <= f3 < f4")
    if f4 > 1.0 / (2.0 * dts):
        raise ValueError("f4 > fNyquist")


def trapezoid(f, f1, f2, f3, f4):
    """Trapezoid amplitude at the frequencies f (waveletFloatMain.py:52-73)."""
    f = np.asarray(f, dtype=np.float64)
    out = np.zeros_like(f)
    up = (f >= f1) & (f < f2)
    out[up] = np.cos(np.pi / 2.0 * (f2 - f[up]) / (f2 - f1)) ** 2
    out[(f >= f2) & (f < f3)] = 1.0
    down = (f >= f3) & (f < f4)
    out[down] = np.cos(np.pi / 2.0 * (f[down] - f3) / (f4 - f3)) ** 2
    return out


def band_wavelet(nts, dts, f1, f2, f3, f4, timeDelay=0.0):
    """Band-limited wavelet of waveletFloatMain.py type "ali" (:13-86).

    The spectrum is built on an even length (nts, or nts + 1 when nts is odd)
    with df = 1 / (length * dts): trapezoid amplitude times the delay phase
    exp(-2 pi i f timeDelay) on bins 0 .. length/2 - 1, zero at Nyquist, the
    conjugate mirror on the negative frequencies.  The wavelet is the real part
    of the inverse FFT (of the first nts bins when nts is odd, as there)."""
    _check_corners(f1, f2, f3, f4, dts)
    n = nts + 1 if nts % 2 else nts
    df = 1.0 / (n * dts)
    f = np.arange(n // 2) * df
    spec = np.zeros(n, np.complex64)
    spec[: n // 2] = (trapezoid(f, f1, f2, f3, f4) * np.exp(-1j * 2.0 * np.pi * f * timeDelay)).astype(np.complex64)
    spec[n // 2 + 1:] = np.flip(spec[1: n // 2].conj(), axis=0)
    sig = np.fft.ifft(spec[:-1] if nts % 2 else spec).real
    return sig.astype(np.float32)


def ricker_wavelet(nts, dts, fDom, timeDelay=0.0, ots=0.0):
    """Ricker wavelet of waveletFloatMain.py type "ricker" (:89-108):
    (1 - 2 a t^2) exp(-a t^2), a = (pi fDom)^2, t = ots + it*dts - timeDelay."""
    alpha = (np.pi * fDom) * (np.pi * fDom)
    t = ots + np.arange(nts) * dts - timeDelay
    return ((1.0 - 2.0 * alpha * t * t) * np.exp(-1.0 * alpha * t * t)).astype(np.float32)


def band_limit(traces, dts, f1, f2, f3, f4, axis=-1):
    """Zero-phase trapezoid filter of real traces along ``axis`` (time):
    the spectrum of each trace is multiplied by the trapezoid amplitude.
    FP64 arithmetic, result in the input's dtype."""
    _check_corners(f1, f2, f3, f4, dts)
    x = np.asarray(traces)
    n = x.shape[axis]
    spec = np.fft.rfft(x.astype(np.float64), axis=axis)
    amp = trapezoid(np.fft.rfftfreq(n, dts), f1, f2, f3, f4)
    shape = [1] * x.ndim
    shape[axis] = amp.size
    out = np.fft.irfft(spec * amp.reshape(shape), n=n, axis=axis)
    return out.astype(x.dtype if np.issubdtype(x.dtype, np.floating) else np.float64)


def multiscale_bands(fmin, fmax, nbands, ramp=1.0):
    """Corner frequencies of a multiscale sequence from fmin to fmax: band k
    keeps [fmin, fk] with fk growing linearly from fmin + (fmax - fmin)/nbands
    to fmax, with cosine ramps of width ``ramp`` Hz on both sides."""
    if not (0.0 < fmin < fmax) or nbands < 1:
        raise ValueError("need 0 < fmin < fmax and nbands >= 1")
    bands = []
    for k in range(1, nbands + 1):
        fk = fmin + (fmax - fmin) * k / nbands
        bands.append((max(fmin - ramp, 0.0), fmin, fk, fk + ramp))
    return bands
