"""Elastic full-waveform inversion around the propagation operators.

The reference drives its FWI (PF/efwiMain.py) with pySolver's nonlinear
solvers, which are not part of the reference tree.  This module supplies the
pieces that script composes, on top of ``nonlinearFwiPropElasticShotsGpu``
(modelling) and ``BornElasticShotsGpu`` (Jacobian):

* ``ElasticDatComp``  -- data-component sampling (SU/python/dataCompModule.py:9-107);
* ``ElasticConv`` / ``ElasticConvJab`` -- parameter conversion VpVsRho <-> RhoLameMu
  and its Jacobian (SU/python/elasticParamConvertModule.py:5-117);
* ``FwiObjective``   -- misfit 0.5 ||S F(m) - d||^2 and its gradient
  J^T S^T (S F(m) - d) through the Born adjoint, with an optional gradient mask
  and bound vectors (efwiMain.py:120-177, 248-256);
* ``lbfgs``          -- limited-memory BFGS with a backtracking (Armijo) line
  search and projection onto the bounds, optionally with learned steps;
* ``band_objective`` / ``multiscale`` -- the multiscale loop of the FWI
  scripts (efwiMain.py is run once per band with band-limited wavelets): the
  objective on band-limited sources and data, and L-BFGS band after band,
  each band starting from the previous band's model.

Reductions that decide the optimisation (misfit, dot products, gradient norm)
run in FP64 on the GPU through the library's own reduction kernels
(``eio_reduce64``: ``dot64``, ``misfit64``); the fields stay FP32.  Without a
visible CUDA device (host-only tests of the solver logic) they are formed in
FP64 with numpy.
"""
import ctypes

import numpy as np

__all__ = ["dot64", "misfit64", "ElasticDatComp", "ElasticConv", "ElasticConvJab", "FwiObjective", "lbfgs",
           "band_objective", "multiscale"]


def _nd(v):
    return v.getNdArray() if hasattr(v, "getNdArray") else v


_HAS_GPU = None


def _gpu():
    global _HAS_GPU
    if _HAS_GPU is None:
        try:
            import torch
            _HAS_GPU = bool(torch.cuda.is_available())
        except ImportError:
            _HAS_GPU = False
    return _HAS_GPU


def _reduce64(op, a, b, device=0):
    a = np.asarray(_nd(a))
    b = a if b is None else np.asarray(_nd(b))
    if a.size != b.size:
        raise ValueError("reduction over arrays of different sizes (%d, %d)" % (a.size, b.size))
    dt = np.float32 if (a.dtype == np.float32 and b.dtype == np.float32) else np.float64
    same = b is a
    a = np.ascontiguousarray(a, dtype=dt)
    b = a if same else np.ascontiguousarray(b, dtype=dt)
    if not _gpu():
        a64, b64 = a.ravel().astype(np.float64), b.ravel().astype(np.float64)
        return float(np.dot(a64, b64)) if op == 0 else float(np.dot(a64 - b64, a64 - b64))
    from . import _lib
    r = ctypes.c_double()
    _lib.check(_lib.lib().eio_reduce64(device, op, 0 if dt == np.float32 else 1, a.ctypes.data, b.ctypes.data,
                                       a.size, 0, ctypes.byref(r)))
    return r.value


def dot64(a, b):
    """FP64 dot product of two arrays (FP32 or FP64 values), summed on the GPU."""
    return _reduce64(0, a, None if b is a else b)


def misfit64(a, b):
    """FP64 sum of (a - b)^2, summed on the GPU."""
    return _reduce64(1, a, b)


# --------------------------------------------------------------------- data components
_COMP = {"vx": 0, "vz": 1, "sxx": 2, "szz": 3, "sxz": 4}


class ElasticDatComp:
    """Sampling of elastic data components: data [nExp][5][nRec][nts] ->
    [nExp][nComp][nRec][nts] for a comma-separated list out of vx, vz, sxx, szz,
    sxz and p = 0.5 (sxx + szz); the adjoint spreads back."""

    def __init__(self, components):
        comps = [c.strip().lower() for c in components.split(",")]
        if len(set(comps)) != len(comps):
            raise ValueError("ERROR! A component was provided multiple times! Check your input arguments")
        if any(c not in _COMP and c != "p" for c in comps):
            raise ValueError("ERROR! Provided unknown data components: %s" % components)
        self.comp_list = comps

    def range_shape(self, domain_shape):
        s = list(domain_shape)
        s[1] = len(self.comp_list)
        return tuple(s)

    def forward(self, add, model, data):
        m, d = _nd(model), _nd(data)
        if not add:
            d[...] = 0.0
        for i, c in enumerate(self.comp_list):
            if c == "p":
                d[:, i] += 0.5 * (m[:, 2] + m[:, 3])
            else:
                d[:, i] += m[:, _COMP[c]]

    def adjoint(self, add, model, data):
        m, d = _nd(model), _nd(data)
        if not add:
            m[...] = 0.0
        for i, c in enumerate(self.comp_list):
            if c == "p":
                m[:, 2] += 0.5 * d[:, i]
                m[:, 3] += 0.5 * d[:, i]
            else:
                m[:, _COMP[c]] += d[:, i]


# --------------------------------------------------------------------- parameter conversion
class ElasticConv:
    """conv_type 1: VpVsRho (m/s, m/s, kg/m3) -> RhoLameMu (kg/m3, Pa, Pa);
    2: the same from km/s, km/s, g/cm3; -1: RhoLameMu -> VpVsRho."""

    def __init__(self, conv_type):
        if conv_type not in (1, 2, -1):
            raise ValueError("ERROR! Unsupported conv_type (current value: %s). Please redefine it!" % conv_type)
        self.conv_type = conv_type

    def forward(self, add, model, data):
        m, d = _nd(model), _nd(data)
        if not add:
            d[...] = 0.0
        if self.conv_type in (1, 2):
            s_rho, s_mod = (1.0, 1.0) if self.conv_type == 1 else (1e3, 1e9)
            d[0] += m[2] * s_rho
            d[1] += m[2] * (m[0] * m[0] - 2.0 * m[1] * m[1]) * s_mod
            d[2] += m[2] * m[1] * m[1] * s_mod
        else:
            d[0] += np.sqrt((m[1] + 2 * m[2]) / m[0])
            d[1] += np.sqrt(m[2] / m[0])
            d[2] += m[0]


class ElasticConvJab:
    """Jacobian of the VpVsRho -> RhoLameMu conversion at ``background``
    (VpVsRho; for conv_type 2 given in km/s, km/s, g/cm3 and scaled like the
    reference's setBackground)."""

    def __init__(self, background, conv_type):
        if conv_type not in (1, 2):
            raise ValueError("ERROR! Unsupported conv_type (current value: %s). Please redefine it!" % conv_type)
        self.conv_type = conv_type
        self.setBackground(background)

    def setBackground(self, background):
        self.bg = np.array(_nd(background), dtype=np.float32, copy=True)
        if self.conv_type == 2:
            self.bg *= 1e3

    def forward(self, add, model, data):
        m, d, b = _nd(model), _nd(data), self.bg
        if not add:
            d[...] = 0.0
        d[0] += m[2]
        d[1] += (b[0] * b[0] - 2.0 * b[1] * b[1]) * m[2] - 4.0 * b[1] * b[2] * m[1] + 2.0 * b[0] * b[2] * m[0]
        d[2] += b[1] * b[1] * m[2] + 2.0 * b[1] * b[2] * m[1]

    def adjoint(self, add, model, data):
        m, d, b = _nd(model), _nd(data), self.bg
        if not add:
            m[...] = 0.0
        m[0] += 2.0 * b[0] * b[2] * d[1]
        m[1] += 2.0 * b[1] * b[2] * d[2] - 4.0 * b[1] * b[2] * d[1]
        m[2] += d[0] + (b[0] * b[0] - 2.0 * b[1] * b[1]) * d[1] + b[1] * b[1] * d[2]


# --------------------------------------------------------------------- objective
class FwiObjective:
    """phi(m) = 0.5 ||S F(m) - d_obs||^2 over the model m [3][nx][nz].

    nl: nonlinearFwiPropElasticShotsGpu (its forward sets m as the background);
    born: BornElasticShotsGpu on the same acquisition (setBackground(m) makes it
    the Jacobian at m); sampler: optional ElasticDatComp S; conv: optional
    ElasticConv (conv_type 1 or 2): m is then VpVsRho and the gradient goes
    through ElasticConvJab^T; mask: optional gradient weights [3][nx][nz].

    fused (default): gradients come from BornElasticShotsGpu.fwiGradient, which
    reuses the source wavefield of the nonlinear forward in the Born adjoint
    (two propagations per shot instead of three; the misfit and gradient agree
    with the unfused evaluation to FP32 rounding).  It needs the Born
    operator's source signals to be the nonlinear operator's sources and no
    free surface; fused=False, or a free surface, takes the unfused path."""

    def __init__(self, nl, born, d_obs, sampler=None, conv=None, mask=None, fused=True):
        self.nl, self.born, self.sampler, self.conv = nl, born, sampler, conv
        self.d_obs = np.asarray(_nd(d_obs), dtype=np.float32)
        self.mask = None if mask is None else np.asarray(_nd(mask), dtype=np.float32)
        self.fused = bool(fused) and hasattr(born, "fwiGradient") and hasattr(nl, "sources") and \
            not getattr(getattr(born, "fd", None), "surfaceCondition", 1)
        self.nfev = 0

    def _elastic(self, m):
        if self.conv is None:
            return np.ascontiguousarray(m, dtype=np.float32)
        out = np.zeros_like(m, dtype=np.float32)
        self.conv.forward(False, m, out)
        return out

    def residual(self, m):
        ep = self._elastic(m)
        dfull = self.nl.dataSpace()
        self.nl.forward(False, ep, dfull)
        d = _nd(dfull)
        if self.sampler is not None:
            ds = np.zeros(self.sampler.range_shape(d.shape), np.float32)
            self.sampler.forward(False, d, ds)
            d = ds
        return ep, d - self.d_obs

    def value(self, m):
        self.nfev += 1
        _, r = self.residual(m)
        return 0.5 * dot64(r, r)

    def value_and_gradient(self, m):
        self.nfev += 1
        if self.fused:
            ep = self._elastic(m)
            comps = None if self.sampler is None else ",".join(self.sampler.comp_list)
            phi, g = self.born.fwiGradient(ep, self.nl.sources, self.d_obs, comps)
        else:
            ep, r = self.residual(m)
            phi = 0.5 * dot64(r, r)
            rfull = r
            if self.sampler is not None:
                rfull = np.zeros(self.nl.dataSpace().getNdArray().shape, np.float32)
                self.sampler.adjoint(False, rfull, r)
            self.born.setBackground(ep)
            g = self.born.modelSpace()
            self.born.adjoint(False, g, np.ascontiguousarray(rfull, dtype=np.float32))
            g = np.array(_nd(g), dtype=np.float32)
        if self.conv is not None:
            jab = ElasticConvJab(m, self.conv.conv_type)
            gm = np.zeros_like(g)
            jab.adjoint(False, gm, g)
            g = gm
        if self.mask is not None:
            g *= self.mask
        return phi, g


# --------------------------------------------------------------------- L-BFGS
def _project(m, lo, hi):
    if lo is not None:
        np.maximum(m, lo, out=m)
    if hi is not None:
        np.minimum(m, hi, out=m)
    return m


def _free(m, g, lo, hi):
    """Variables not held at a bound by the gradient (the active set is frozen)."""
    free = np.ones(m.shape, dtype=bool)
    if lo is not None:
        free &= ~((m <= lo) & (g > 0))
    if hi is not None:
        free &= ~((m >= hi) & (g < 0))
    return free


class _Scaled:
    """objective of x = m / scale (elementwise): value(x) = phi(x * scale),
    gradient = scale * dphi/dm."""

    def __init__(self, objective, scale):
        self.obj, self.scale = objective, scale

    def value(self, x):
        return self.obj.value((x * self.scale).astype(np.float32))

    def value_and_gradient(self, x):
        f, g = self.obj.value_and_gradient((x * self.scale).astype(np.float32))
        return f, (g * self.scale).astype(np.float32)


def lbfgs(objective, m0, niter=10, memory=5, minBound=None, maxBound=None, init_step=None, c1=1e-4,
          max_backtrack=8, callback=None, scale=None, precond=None, stats=None):
    """Minimise ``objective``; with ``scale`` (an array of m's shape, e.g. the
    starting model) the search runs on m / scale so that parameters of very
    different units weigh alike.  ``precond(m, g)`` (e.g. a
    precond.LearnedPreconditioner) proposes a model update that is tried before
    each L-BFGS step and kept only when the exact misfit accepts it; ``stats``
    (a dict) receives the counts of accepted and rejected learned steps.  See
    _lbfgs for the method."""
    if scale is None:
        return _lbfgs(objective, m0, niter, memory, minBound, maxBound, init_step, c1, max_backtrack, callback,
                      precond, stats)
    sc = np.where(np.asarray(scale) != 0, np.asarray(scale), 1.0).astype(np.float32)
    lo = None if minBound is None else minBound / sc
    hi = None if maxBound is None else maxBound / sc
    if lo is not None and hi is not None:
        lo, hi = np.minimum(lo, hi), np.maximum(lo, hi)
    cb = None if callback is None else (lambda it, x, f, g: callback(it, x * sc, f, g / sc))
    pc = None if precond is None else (lambda x, gx: precond((x * sc).astype(np.float32), gx / sc) / sc)
    x, hist = _lbfgs(_Scaled(objective, sc), np.asarray(m0) / sc, niter, memory, lo, hi, init_step, c1,
                     max_backtrack, cb, pc, stats)
    return (x * sc).astype(np.float32), hist


def _trial_value(objective, mt):
    """Misfit at a trial point of a line search; +inf when the propagator's
    stability or dispersion check refuses the model (the search backtracks)."""
    from ._lib import EioError
    try:
        return objective.value(mt)
    except EioError as e:
        if e.code != -2:              # anything but a refused model is an error
            raise
        return np.inf


def _two_loop(g, free, S, Y, rho, h0):
    """L-BFGS direction -H g on the free variables: the two-loop recursion over
    the stored pairs around the initial inverse Hessian h0 (a function)."""
    q = np.where(free, g, 0).astype(np.float64)
    alpha = []
    for s, y, r in reversed(list(zip(S, Y, rho))):
        a = r * dot64(s, q)
        alpha.append(a)
        q = q - a * y
    q = np.asarray(h0(q), dtype=np.float64)
    for (s, y, r), a in zip(zip(S, Y, rho), reversed(alpha)):
        b = r * dot64(y, q)
        q = q + (a - b) * s
    return np.where(free, -q, 0)


def _max_rel(d, m):
    am = np.abs(m).astype(np.float64)
    return float((np.abs(d) / np.where(am > 0, am, max(float(am.max()), 1e-30))).max())


def _lbfgs(objective, m0, niter=10, memory=5, minBound=None, maxBound=None, init_step=None, c1=1e-4,
           max_backtrack=8, callback=None, precond=None, stats=None, max_rel=0.1, learned_c1=0.2):
    """Minimise ``objective`` (value_and_gradient(m), value(m)) from m0.

    Two-loop recursion over the last ``memory`` pairs on the variables that no
    bound holds (an active-set restriction keeps the direction a descent one
    for the projected problem); the first step, and every step after a restart,
    is scaled so that no model value changes by more than ``init_step`` of
    itself (default 1 %); trial points are projected onto [minBound,
    maxBound]; backtracking halves the step until the Armijo condition holds
    (a model the propagator's checks refuse counts as a failed trial), and a
    failed search restarts once from the projected steepest descent.
    With ``precond`` (a learned approximate inverse Hessian, precond(m, g) ~
    -H^-1 g), the recursion runs around it, scaled by the latest curvature
    pair, instead of the scalar initial Hessian; the exact misfit decides the
    step (sufficient decrease with learned_c1, two trials), and when it
    rejects the learned direction, or that is no descent direction, the
    iteration falls back to the plain L-BFGS step.
    Returns (m, history) with history the objective values (FP64)."""
    m = _project(np.array(m0, dtype=np.float32, copy=True), minBound, maxBound)
    f, g = objective.value_and_gradient(m)
    hist = [f]
    S, Y, rho = [], [], []
    it = 0
    restarted = False
    if stats is not None:
        stats.setdefault("learned", 0)
        stats.setdefault("rejected", 0)
    plain_only = False
    while it < niter:
        free = _free(m, g, minBound, maxBound)
        learned = False
        d = None
        if precond is not None and not plain_only:
            # the learned operator as the initial inverse Hessian, scaled by the
            # latest curvature pair (gamma = s.y / y.P y, P = -precond) once
            # there is one; the search starts at the full step, capped at a
            # max_rel relative change of any model value
            def P(q):
                return -np.asarray(precond(m, np.asarray(q, np.float32)), np.float64)
            gamma = 1.0
            if S:
                yPy = dot64(Y[-1], P(Y[-1]))
                if yPy > 0:
                    gamma = dot64(S[-1], Y[-1]) / yPy
            d = _two_loop(g, free, S, Y, rho, lambda q: gamma * P(q))
            if np.isfinite(d).all() and d.any() and dot64(g, d) < 0:
                learned = True
                step = min(1.0, max_rel / max(_max_rel(d, m), 1e-300)) if not S else 1.0
            else:
                d = None
                if stats is not None:
                    stats["rejected"] += 1
        plain_only = False
        if d is None:
            d = _two_loop(g, free, S, Y, rho,
                          lambda q: q * (dot64(S[-1], Y[-1]) / dot64(Y[-1], Y[-1])) if S else q)
            if dot64(g, d) >= 0:  # not a descent direction: restart from steepest descent
                S, Y, rho = [], [], []
                d = np.where(free, -g, 0).astype(np.float64)
            if not S:
                # parameters of very different scales (kg/m3 and Pa): bound the
                # largest relative change of any model value by init_step
                frac = 0.01 if init_step is None else init_step
                step = frac / max(_max_rel(d, m), 1e-300)
            else:
                step = 1.0
        accepted = False
        # a learned step must deliver a fifth of the decrease its slope
        # predicts (a Newton step on a quadratic delivers half), within two
        # trials; a plain step the Armijo condition with c1
        cl = learned_c1 if learned else c1
        for _ in range(2 if learned else max_backtrack + 1):
            mt = _project((m + step * d).astype(np.float32), minBound, maxBound)
            ft = _trial_value(objective, mt)
            if ft <= f + cl * dot64(g, mt - m) and ft < f:
                accepted = True
                break
            step *= 0.5
        if not accepted and learned:
            # the exact misfit rejected the learned direction: plain step instead
            if stats is not None:
                stats["rejected"] += 1
            plain_only = True
            continue
        if learned and stats is not None:
            stats["learned"] += 1
        if not accepted:
            if S and not restarted:
                S, Y, rho = [], [], []
                restarted = True
                continue
            break
        restarted = False
        ft, gt = objective.value_and_gradient(mt)
        s = (mt - m).astype(np.float64)
        y = (gt - g).astype(np.float64)
        sy = dot64(s, y)
        if sy > 1e-10 * np.sqrt(dot64(s, s) * dot64(y, y)):
            S.append(s); Y.append(y); rho.append(1.0 / sy)
            if len(S) > memory:
                S.pop(0); Y.pop(0); rho.pop(0)
        m, f, g = mt, ft, gt
        hist.append(f)
        if callback is not None:
            callback(it, m, f, g)
        it += 1
    return m, hist


# --------------------------------------------------------------------- multiscale
def band_objective(nl, born, d_obs, sources, dts, band, **objective_kw):
    """FwiObjective of one frequency band: the source traces ``sources`` (the
    nonlinear FWI operator's, [nModelExp][5][nSrc][nts]) and the observed data
    filtered with the zero-phase trapezoid ``band`` = (f1, f2, f3, f4)
    (wavelet.band_limit); both operators get the filtered sources.

    ``nl.sources`` holds the filtered traces afterwards.  The first call keeps
    a copy of the broadband traces the operator was built with
    (``nl._broadband_sources``); passing ``sources=None`` or ``nl.sources``
    itself filters that copy, so a band loop never filters traces that an
    earlier band already filtered."""
    from .wavelet import band_limit
    if not hasattr(nl, "_broadband_sources"):
        nl._broadband_sources = np.array(_nd(nl.sources), dtype=np.float32, copy=True)
    if sources is None or sources is nl.sources:
        src = nl._broadband_sources
    else:
        src = np.asarray(_nd(sources), dtype=np.float32)
    src_b = band_limit(src, dts, *band, axis=-1).astype(np.float32)
    d_b = band_limit(np.asarray(_nd(d_obs), dtype=np.float32), dts, *band, axis=-1).astype(np.float32)
    nl.sources = np.ascontiguousarray(src_b)
    per = src_b.reshape(-1, *src_b.shape[-3:])
    born.setSourceSignals([per[i] for i in range(per.shape[0])])
    return FwiObjective(nl, born, d_b, **objective_kw)


def multiscale(objective_for_band, m0, bands, niter=10, callback=None, iter_callback=None, **lbfgs_kw):
    """L-BFGS band after band: ``objective_for_band(band)`` gives the objective
    of a band (e.g. band_objective), each band starts from the model the
    previous one reached.  ``callback(k, band, m, history)`` after each band;
    ``iter_callback(k, it, m, f, g)`` after each iteration of band k (the
    L-BFGS callback).  Returns (m, [history of each band])."""
    m = np.array(m0, dtype=np.float32, copy=True)
    hists = []
    for k, band in enumerate(bands):
        obj = objective_for_band(band)
        cb = None if iter_callback is None else (lambda it, mm, f, g, k=k: iter_callback(k, it, mm, f, g))
        m, hist = lbfgs(obj, m, niter=niter, callback=cb, **lbfgs_kw)
        hists.append(hist)
        if callback is not None:
            callback(k, band, m, hist)
    return m, hists
