"""Seeded synthetic media, wavelets and acquisitions of the benchmark workloads.

* ``pad_elastic`` restates padElasticFileGpuMain (edge replication to zPad/xPad,
  the plus-side pad grown so that the padded size is a multiple of blockSize,
  then a FAT frame), elastic_iso_lib/seis_utils/seis_utils_float/src/padElasticFileGpuMain.cpp:26-159.
* ``ricker`` restates the Ricker branch of waveletFloatMain.py:88-108.
* ``gardner``: rho = 310 vp^0.25 (kg/m^3, vp in m/s).

Workloads (all seeded, no external data):
  nl_312x520     200x400 interior + 50-cell pads (312x520 total), dx=dz=10 m,
                 dt=1 ms, nts=2000, 6 flat layers vp 1500..3500 m/s, vs=vp/sqrt(3)
                 (0 in the water layer), Gardner rho, 15 Hz Ricker explosive
                 source at z=20 m, 400 receivers at z=20 m
  born_600x1800  600x1800 total (50-cell pads), dx=dz=10 m, dt=0.8 ms, nts=4000,
                 vp gradient 1800..4000 m/s, vs=vp/1.8, Gardner rho, seeded
                 Gaussian-random drho/dlambda/dmu smoothed at 50 m with 5% RMS,
                 10 shots (12 Hz Ricker), 900 receivers
  fwi_1000x3400  batched FWI gradient: 1000x3400 total (50-cell pads), dx=dz=12.5 m,
                 dt=1 ms, nts=5000, flat layers vp 1800..4000 m/s with a seeded
                 irregular 4500 m/s inclusion (true model) and its Gaussian-smoothed
                 version (starting model), vs=vp/1.8, Gardner rho, 10 Hz Ricker,
                 120 shots whose receivers (same count) span an offset window of
                 2..8 km drawn per shot (uneven apertures, so cropped windows differ)
  small          tiny grid for parity tests
"""
import math

import numpy as np

from . import padding

from .sepvec import axis, hypercube, floatVector, paramObj

FAT = 4


def gardner(vp):
    return 310.0 * np.power(vp, 0.25)


def elastic_from_vpvsrho(vp, vs, rho):
    """(rho, lambda, mu) stacked as [3][nx][nz] from [nx][nz] vp, vs, rho."""
    mu = rho * vs * vs
    lam = rho * vp * vp - 2.0 * mu
    return np.stack([rho, lam, mu]).astype(np.float32)


def pad_elastic(ep, zPad, xPad, fat=FAT, blockSize=16):
    """ep: [npar][nx][nz] -> padded array and the pad sizes (surfaceCondition = 0)."""
    return padding.pad_elastic_array(ep, zPad, xPad, fat, blockSize, 0)


def ricker(nts, dts, fdom, delay, ots=0.0):
    t = ots + np.arange(nts) * dts - delay
    a = (np.pi * fdom) ** 2
    return ((1.0 - 2.0 * a * t * t) * np.exp(-a * t * t)).astype(np.float32)


def gaussian_smooth(f, sigma_cells):
    """Separable Gaussian smoothing (truncated at 4 sigma, reflect edges)."""
    r = int(math.ceil(4 * sigma_cells))
    k = np.exp(-0.5 * (np.arange(-r, r + 1) / sigma_cells) ** 2)
    k /= k.sum()
    out = f.astype(np.float64)
    for ax in range(out.ndim):
        pad = [(0, 0)] * out.ndim
        pad[ax] = (r, r)
        p = np.pad(out, pad, mode="reflect")
        out = np.apply_along_axis(lambda v: np.convolve(v, k, mode="valid"), ax, p)
    return out


def elastic_vector(ep, oz, ox, dz, dx):
    h = hypercube(axes=[axis(ep.shape[2], oz, dz), axis(ep.shape[1], ox, dx), axis(3)])
    return floatVector(h, ep)


class Workload:
    """Medium, parameters and acquisition of one synthetic case."""

    def __init__(self, name, ep, pads, dz, dx, nts, dts, sub, fMax, src_z, src_x, rec_z, rec_x, wavelet,
                 nExp, extra=None):
        self.name = name
        nz, nx = ep.shape[2], ep.shape[1]
        self.oz = -(FAT + pads["zPadMinus"]) * dz
        self.ox = -(FAT + pads["xPadMinus"]) * dx
        self.elastic = elastic_vector(ep, self.oz, self.ox, dz, dx)
        self.par = paramObj(dict(nts=nts, dts=dts, ots=0.0, sub=sub, nz=nz, nx=nx, dz=dz, dx=dx, fMax=fMax,
                                 blockSize=16, fat=FAT, alphaCos=0.99, nExp=nExp, **pads))
        self.nz, self.nx, self.nts, self.dts, self.sub = nz, nx, nts, dts, sub
        self.dz, self.dx = dz, dx
        self.src_z = np.asarray(src_z, np.float32)   # [nExp] physical coordinates of the padded grid frame
        self.src_x = np.asarray(src_x, np.float32)
        self.rec_z = np.asarray(rec_z, np.float32)
        self.rec_x = np.asarray(rec_x, np.float32)
        self.wavelet = wavelet
        self.nExp = nExp
        self.extra = extra or {}

    @property
    def ntw(self):
        return (self.nts - 1) * 2 * self.sub + 1

    @property
    def cells(self):
        return (self.nz - 2 * FAT) * (self.nx - 2 * FAT)

    @property
    def fine_steps(self):
        return (self.nts - 1) * 2 * self.sub

    def source_signal(self):
        """Explosive source: the wavelet in sigmaxx and sigmazz; [5][1][nts]."""
        s = np.zeros((5, 1, self.nts), np.float32)
        s[2, 0] = self.wavelet
        s[3, 0] = self.wavelet
        return s

    def geometry(self, method="linear", nfilt=1):
        """Four staggered-grid interpolators per shot (prop.spaceInterpGpu)."""
        from .prop import spaceInterpGpu, _staggered_hypers
        hyps = _staggered_hypers(self.elastic)
        src = [[], [], [], []]
        for e in range(self.nExp):
            zc = self.src_z[e:e + 1].copy()
            xc = self.src_x[e:e + 1].copy()
            for k, h in enumerate(hyps):
                src[k].append(spaceInterpGpu(zc, xc, h, self.nts, method, nfilt, 0, 0.0, 0.0))
        if "rec_x_shots" in self.extra:   # per-shot receivers (same count, own positions)
            rec = [[spaceInterpGpu(np.full(len(rx), self.rec_z[0], np.float32), np.asarray(rx, np.float32), h,
                                   self.nts, method, nfilt, 0, 0.0, 0.0) for rx in self.extra["rec_x_shots"]]
                   for h in hyps]
            return src, rec
        rec = [[spaceInterpGpu(self.rec_z, self.rec_x, h, self.nts, method, nfilt, 0, 0.0, 0.0)] for h in hyps]
        return src, rec


def _grid_coord(o, d, idx):
    return np.float32(o + idx * d)


def nl_312x520(nts=2000, nshots=1):
    """Plain nonlinear modelling case: 200x400 interior with 50-cell pads, six
    flat layers, 15 Hz Ricker at 20 m depth, 400 receivers.  nshots > 1 spreads
    further sources along the line (the first one stays mid-line)."""
    nzi, nxi, dz = 200, 400, 10.0
    vps = np.array([1500, 1900, 2300, 2700, 3100, 3500], np.float64)
    layer = np.minimum((np.arange(nzi) * len(vps)) // nzi, len(vps) - 1)
    vp = np.tile(vps[layer], (nxi, 1))
    vs = vp / math.sqrt(3.0)
    vs[:, layer == 0] = 0.0
    ep = elastic_from_vpvsrho(vp, vs, gardner(vp))
    epp, pads = pad_elastic(ep, 50, 50)
    dts = 1e-3
    oz = -(FAT + 50) * dz
    ox = -(FAT + 50) * dz
    # z = 20 m below the top of the interior; source mid-line
    z0 = _grid_coord(oz, dz, FAT + 50 + 2)
    cols = [nxi // 2] + [int(round(c)) for c in np.linspace(20, nxi - 21, max(nshots - 1, 1))][:nshots - 1]
    src_x = [_grid_coord(ox, dz, FAT + 50 + c) for c in cols]
    rec_x = np.array([_grid_coord(ox, dz, FAT + 50 + i) for i in range(nxi)], np.float32)
    rec_z = np.full(nxi, z0, np.float32)
    w = ricker(nts, dts, 15.0, 0.1)
    return Workload("nl_312x520", epp, pads, dz, dz, nts, dts, 1, 30.0, [z0] * nshots, src_x, rec_z, rec_x, w,
                    nshots)


def born_600x1800(nts=4000, nshots=10, seed=2024, select=None):
    """Born benchmark case: 600x1800 grid (50-cell pads), vp gradient
    1800-4000 m/s, vs = vp/1.8, Gardner density, seeded smoothed 5 % RMS
    perturbations of rho, lambda, mu, nshots 12 Hz Ricker shots spread over the
    line, 900 receivers centred on it.  select: indices of the shots to keep."""
    nz, nx, dz = 600, 1800, 10.0
    pad = 50
    nzi, nxi = nz - 2 * FAT - 2 * pad, nx - 2 * FAT - 2 * pad
    depth = np.arange(nzi) / (nzi - 1)
    vp = np.tile(1800.0 + (4000.0 - 1800.0) * depth, (nxi, 1))
    vs = vp / 1.8
    ep = elastic_from_vpvsrho(vp, vs, gardner(vp))
    epp, pads = pad_elastic(ep, pad, pad)
    assert epp.shape == (3, nx, nz), epp.shape
    rng = np.random.default_rng(seed)
    dmod = np.zeros_like(epp)
    for k in range(3):
        f = gaussian_smooth(rng.standard_normal((nx, nz)), 5.0)
        f = f / np.sqrt(np.mean(f * f))
        dmod[k] = (0.05 * np.sqrt(np.mean(epp[k].astype(np.float64) ** 2)) * f).astype(np.float32)
    dts = 0.8e-3
    oz = -(FAT + pad) * dz
    ox = -(FAT + pad) * dz
    z0 = _grid_coord(oz, dz, FAT + pad + 2)
    xs = np.linspace(FAT + pad + 20, FAT + pad + nxi - 21, nshots).round().astype(int)
    if select is not None:
        xs = xs[list(select)]
        nshots = len(xs)
    src_x = [_grid_coord(ox, dz, i) for i in xs]
    first = FAT + pad + (nxi - 900) // 2
    rec_x = np.array([_grid_coord(ox, dz, first + i) for i in range(900)], np.float32)
    rec_z = np.full(900, z0, np.float32)
    w = ricker(nts, dts, 12.0, 0.12)
    return Workload("born_600x1800", epp, pads, dz, dz, nts, dts, 1, 30.0, [z0] * nshots, src_x, rec_z, rec_x,
                    w, nshots, extra=dict(dmodel=dmod))


def fwi_1000x3400(nts=5000, nshots=120, nrec=200, seed=2025, nz=1000, nx=3400, dz=12.5, pad=50,
                  window_km=(2.0, 8.0), select=None):
    """Batched-FWI case (see the module docstring); other sizes for tests.
    select: indices of the shots to keep (the acquisition of the others is drawn
    all the same, so a subset is the same shots as in the full case).
    extra: true_model / start_model ([3][nx][nz] padded), rec_x_shots."""
    nzi, nxi = nz - 2 * FAT - 2 * pad, nx - 2 * FAT - 2 * pad
    rng = np.random.default_rng(seed)
    depth = np.arange(nzi) / max(nzi - 1, 1)
    layers = np.array([1800, 2100, 2400, 2700, 3000, 3300, 3600, 4000], np.float64)
    vp0 = np.tile(layers[np.minimum((depth * len(layers)).astype(int), len(layers) - 1)], (nxi, 1))
    blob = gaussian_smooth(rng.standard_normal((nxi, nzi)), max(nzi, nxi) / 40.0)
    xx, zz = np.meshgrid(np.arange(nxi) / nxi, depth, indexing="ij")
    inside = (blob > 0.2 * blob.std()) & ((xx - 0.5) ** 2 / 0.06 + (zz - 0.55) ** 2 / 0.04 < 1.0)
    vp_true = np.where(inside, 4500.0, vp0)
    vp_start = gaussian_smooth(vp_true, max(nzi, nxi) / 60.0)
    models = []
    for vp in (vp_true, vp_start):
        ep = elastic_from_vpvsrho(vp, vp / 1.8, gardner(vp))
        epp, pads = pad_elastic(ep, pad, pad)
        assert epp.shape == (3, nx, nz), epp.shape
        models.append(epp)
    dts = 1e-3
    oz = -(FAT + pad) * dz
    ox = -(FAT + pad) * dz
    z0 = _grid_coord(oz, dz, FAT + pad + 2)
    first, last = FAT + pad + 10, FAT + pad + nxi - 11
    xs = np.linspace(first, last, nshots).round().astype(int)
    src_x = [_grid_coord(ox, dz, i) for i in xs]
    rec_shots = []
    for i in xs:
        half = 0.5 * rng.uniform(*window_km) * 1000.0 / dz            # cells
        lo, hi = max(first, int(round(i - half))), min(last, int(round(i + half)))
        rec_shots.append(np.array([_grid_coord(ox, dz, c) for c in np.linspace(lo, hi, nrec)], np.float32)
                         + np.float32(0.5 * dz))
    if select is not None:
        src_x = [src_x[i] for i in select]
        rec_shots = [rec_shots[i] for i in select]
    n = len(src_x)
    w = ricker(nts, dts, 10.0, 0.15)
    wl = Workload("fwi_%dx%d" % (nz, nx), models[1], pads, dz, dz, nts, dts, 1, 20.0, [z0] * n, src_x,
                  np.full(nrec, z0, np.float32), rec_shots[0], w, n,
                  extra=dict(true_model=models[0], start_model=models[1], rec_x_shots=rec_shots))
    return wl


def small(nz=72, nx=104, nts=150, nshots=2, nrec=20, seed=7, sub=1, dz=10.0, surface=0, alphaCos=0.99):
    """Tiny layered case (parity tests): pads 12, random smooth perturbation.
    surface = 1: free surface at the top (padding rule of padElasticFileGpuMain
    with surfaceCondition = 1: a fat-cell top pad), devices a few cells below it."""
    pad = 12
    rng = np.random.default_rng(seed)
    ztop = FAT if surface else pad
    nzi, nxi = nz - 2 * FAT - ztop - pad, nx - 2 * FAT - 2 * pad
    assert nzi > 0 and nxi > 0
    depth = np.arange(nzi) / max(nzi - 1, 1)
    vp = np.tile(2000.0 + 1000.0 * depth, (nxi, 1)) + 100.0 * rng.standard_normal((nxi, nzi)).clip(-2, 2)
    vs = vp / 1.7
    ep = elastic_from_vpvsrho(vp, vs, gardner(vp))
    epp, pads = padding.pad_elastic_array(ep, pad, pad, FAT, 16, surface)
    assert epp.shape == (3, nx, nz), (epp.shape, nx, nz)
    dts = 1e-3
    oz = -(FAT + pads["zPadMinus"]) * dz
    ox = -(FAT + pad) * dz
    z0 = _grid_coord(oz, dz, FAT + pads["zPadMinus"] + 2) + np.float32(3.0)   # off-grid: exercises bilinear weights
    src_x = [_grid_coord(ox, dz, FAT + pad + 5 + 7 * e) + np.float32(4.0) for e in range(nshots)]
    rec_x = np.array([_grid_coord(ox, dz, FAT + pad + 2 + i * max(nxi - 4, 1) // nrec) + np.float32(2.5)
                      for i in range(nrec)], np.float32)
    rec_z = np.full(nrec, z0 + np.float32(20.0), np.float32)
    w = ricker(nts, dts, 10.0, 0.06)
    dmod = np.zeros_like(epp)
    for k in range(3):
        f = gaussian_smooth(rng.standard_normal((nx, nz)), 2.0)
        f = f / np.sqrt(np.mean(f * f))
        dmod[k] = (0.05 * np.sqrt(np.mean(epp[k].astype(np.float64) ** 2)) * f).astype(np.float32)
    wl = Workload("small", epp, pads, dz, dz, nts, dts, sub, 25.0, [z0] * nshots, src_x, rec_z, rec_x, w,
                  nshots, extra=dict(dmodel=dmod))
    wl.par.set("surfaceCondition", str(int(surface)))
    wl.par.set("alphaCos", str(alphaCos))
    return wl
