"""CPU oracle for the elastic propagation path -- TEST INFRASTRUCTURE.

Only tests/, __graft_entry__.smoke() and bench.py (cpu_baseline and the
reference arm) may import this module, and only as the checker or the timed
CPU baseline; the product package never imports it.

Two layers:
* ``Oracle(prec)``: ctypes binding of liborc.so (oracle_impl.h restated in
  float ``'f'`` or double ``'d'``): constants, medium preparation, staggering,
  time/space interpolation and the four single-shot propagations on the
  regular grid (propShotsElasticFwdGpu / ...AdjGpu, BornShotsFwdGpu / ...AdjGpu).
* operator level in numpy (``nl_forward`` ...): the per-shot host preparation
  of nonlinearPropElasticGpu.cpp:43-473, seismicElasticOperator2D.cpp:27-117
  and the multi-shot loops of nonlinearPropElasticShotsGpu.cpp:80-422 /
  BornElasticShotsGpu.cpp:85-378 (paths relative to
  elastic_iso_lib/elastic_iso_float/prop of the reference project).
* ``RefGpu(prec)``: the reference's own CUDA driver layer compiled from the
  reference tree into oracle/_ref (oracle/ref/Makefile); same call signature
  as ``Oracle.nl_prop`` / ``Oracle.born_prop``.  Needs a GPU.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liborc.so")
REF_DIR = os.path.join(HERE, "_ref")
FIELD_GRID = (1, 2, 0, 0, 3)   # vx->x, vz->z, sxx/szz->center, sxz->xz
METHODS = {"linear": 0, "sinc": 1, "gauss": 2}

_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        _lib = ctypes.CDLL(LIB)
    return _lib


def num_threads():
    return int(_load().orc_num_threads())


def _pp(arrs, ctype):
    """array of pointers to the given numpy arrays"""
    out = (ctypes.c_void_p * len(arrs))()
    for i, a in enumerate(arrs):
        out[i] = a.ctypes.data if a is not None and a.size else None
    return out


class Oracle:
    def __init__(self, prec="f"):
        assert prec in ("f", "d")
        self.prec = prec
        self.dt = np.float32 if prec == "f" else np.float64
        self.L = _load()
        self.R = ctypes.c_float if prec == "f" else ctypes.c_double

    def _fn(self, name):
        return getattr(self.L, "%s_%s" % (name, self.prec))

    def _a(self, x):
        return np.ascontiguousarray(x, dtype=self.dt)

    # ---------------------------------------------------------------- small pieces
    def consts(self, nz, nx, dz, dx, nts, dts, S, minPad, alphaCos):
        zc = np.zeros(4, self.dt); xc = np.zeros(4, self.dt)
        filt = np.zeros(2 * (S + 1), self.dt); damp = np.zeros(max(minPad, 1), self.dt)
        f = self._fn("orc_consts")
        f.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_float, ctypes.c_int, ctypes.c_float,
                      ctypes.c_int, ctypes.c_int, ctypes.c_float] + [ctypes.c_void_p] * 4
        r = f(nz, nx, dz, dx, nts, dts, S, minPad, alphaCos, zc.ctypes.data, xc.ctypes.data, filt.ctypes.data,
              damp.ctypes.data)
        assert r == 0
        return zc, xc, filt, damp[:minPad]

    def medium(self, ep, dts, S):
        ep = self._a(ep)
        nx, nz = ep.shape[1], ep.shape[2]
        out = [np.zeros((nx, nz), self.dt) for _ in range(5)]
        f = self._fn("orc_medium")
        f.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_int] + [ctypes.c_void_p] * 6
        assert f(nz, nx, dts, S, ep.ctypes.data, *[o.ctypes.data for o in out]) == 0
        return out

    def stagger(self, axis_, adj, add, model, data):
        nx, nz = model.shape
        f = self._fn("orc_stagger_x" if axis_ == 0 else "orc_stagger_z")
        f.argtypes = [ctypes.c_int] * 4 + [ctypes.c_void_p] * 2
        f(adj, add, nz, nx, model.ctypes.data, data.ctypes.data)

    def tinterp(self, adj, add, nts, dts, ots, S, coarse, fine):
        f = self._fn("orc_tinterp")
        f.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_float, ctypes.c_int,
                      ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
        f(adj, add, nts, dts, ots, S, coarse.shape[0], coarse.ctypes.data, fine.ctypes.data)

    def sinterp(self, zc, xc, nz, oz, dz, nx, ox, dx, method="linear", nfilt=1, dipole=0, zds=0.0, xds=0.0):
        """Weights/positions of spaceInterpGpu: returns dict(slot, w, uniq, nft)."""
        zc = self._a(np.ravel(zc)); xc = self._a(np.ravel(xc))
        nd = zc.size
        m = METHODS[method]
        nf = 1 if m == 0 else nfilt
        cap = nd * max(8, (2 * nf) ** 2)
        gpi = np.zeros(cap, np.int32); w = np.zeros(cap, self.dt); slot = np.zeros(cap, np.int32)
        uniq = np.zeros(cap, np.int32); nu = ctypes.c_int(); nft = ctypes.c_int()
        f = self._fn("orc_sinterp_build")
        f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_float,
                      ctypes.c_int, ctypes.c_float, ctypes.c_float, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                      ctypes.c_float, ctypes.c_float] + [ctypes.c_void_p] * 6
        r = f(zc.ctypes.data, xc.ctypes.data, nd, nz, oz, dz, nx, ox, dx, m, nfilt, dipole, zds, xds,
              gpi.ctypes.data, w.ctypes.data, slot.ctypes.data, uniq.ctypes.data, ctypes.byref(nu),
              ctypes.byref(nft))
        if r != 0:
            raise ValueError("oracle sinterp failed (%d)" % r)
        n = nd * nft.value
        return dict(gpi=gpi[:n], w=w[:n], slot=slot[:n], uniq=uniq[:nu.value].copy(), nft=nft.value, nIrreg=nd)

    def sinterp_apply(self, s, adj, add, reg, irreg):
        f = self._fn("orc_sinterp_apply")
        f.argtypes = [ctypes.c_int] * 6 + [ctypes.c_void_p] * 4
        f(adj, add, s["nIrreg"], s["nft"], len(s["uniq"]), reg.shape[1], s["slot"].ctypes.data,
          s["w"].ctypes.data, reg.ctypes.data, irreg.ctypes.data)

    # ---------------------------------------------------------------- propagation
    def nl_prop(self, adj, g, medium5, model5, data5, srcPos, recPos, wavefield=None):
        """g: dict(nz, nx, dz, dx, nts, dts, S, minPad, alphaCos).  model5/data5: lists of
        [nPts][nts] arrays of self.dt (output ones are overwritten).  wavefield: None or a
        [nts][5][nx][nz] array of self.dt, overwritten with the saved wavefield."""
        f = self._fn("orc_nl_prop_fs")
        f.argtypes = [ctypes.c_int] * 3 + [ctypes.c_float] * 2 + [ctypes.c_int, ctypes.c_float, ctypes.c_int,
                                                                   ctypes.c_int, ctypes.c_float] + \
            [ctypes.c_void_p] * 8 + [ctypes.c_int]
        wp = None if wavefield is None else wavefield.ctypes.data
        ns = (ctypes.c_int * 4)(*[len(p) for p in srcPos])
        nr = (ctypes.c_int * 4)(*[len(p) for p in recPos])
        sp = [np.ascontiguousarray(p, np.int32) for p in srcPos]
        rp = [np.ascontiguousarray(p, np.int32) for p in recPos]
        if wavefield is not None:
            assert wavefield.dtype == self.dt and wavefield.flags["C_CONTIGUOUS"]
            assert wavefield.shape == (g["nts"], 5, g["nx"], g["nz"])
        r = f(adj, g["nz"], g["nx"], g["dz"], g["dx"], g["nts"], g["dts"], g["S"], g["minPad"], g["alphaCos"],
              _pp(medium5, None), _pp(model5, None), _pp(data5, None), _pp(sp, None), ns, _pp(rp, None), nr, wp,
              int(g.get("surface", 0)))
        assert r == 0, r

    def born_prop(self, adj, g, medium5, srcDtw5, dm5, data5, srcPos, recPos):
        f = self._fn("orc_born_prop")
        f.argtypes = [ctypes.c_int] * 3 + [ctypes.c_float] * 2 + [ctypes.c_int, ctypes.c_float, ctypes.c_int,
                                                                   ctypes.c_int, ctypes.c_float] + [ctypes.c_void_p] * 8
        ns = (ctypes.c_int * 4)(*[len(p) for p in srcPos])
        nr = (ctypes.c_int * 4)(*[len(p) for p in recPos])
        sp = [np.ascontiguousarray(p, np.int32) for p in srcPos]
        rp = [np.ascontiguousarray(p, np.int32) for p in recPos]
        r = f(adj, g["nz"], g["nx"], g["dz"], g["dx"], g["nts"], g["dts"], g["S"], g["minPad"], g["alphaCos"],
              _pp(medium5, None), _pp(srcDtw5, None), _pp(dm5, None), _pp(data5, None), _pp(sp, None), ns,
              _pp(rp, None), nr)
        assert r == 0, r


class RefGpu:
    """The reference's own CUDA drivers (oracle/_ref, built from the reference tree)."""

    def __init__(self, prec="f"):
        self.prec = prec
        self.dt = np.float32 if prec == "f" else np.float64
        R = ctypes.c_float if prec == "f" else ctypes.c_double
        self.nl = ctypes.CDLL(os.path.join(REF_DIR, "libref_nl_%s.so" % prec))
        self.born = ctypes.CDLL(os.path.join(REF_DIR, "libref_born_%s.so" % prec))
        self.nl.ref_nl_prop.argtypes = [ctypes.c_int] * 3 + [R] * 2 + [ctypes.c_int, R, ctypes.c_int, ctypes.c_int,
                                                                       R] + [ctypes.c_void_p] * 7 + [ctypes.c_int]
        self.born.ref_born_prop.argtypes = [ctypes.c_int] * 3 + [R] * 2 + [ctypes.c_int, R, ctypes.c_int,
                                                                           ctypes.c_int, R] + [ctypes.c_void_p] * 8
        self.nl.ref_nl_prop_wf.argtypes = [ctypes.c_int] * 3 + [R] * 2 + [ctypes.c_int, R, ctypes.c_int,
                                                                          ctypes.c_int, R] + [ctypes.c_void_p] * 8

    @staticmethod
    def available(prec="f"):
        return all(os.path.exists(os.path.join(REF_DIR, "libref_%s_%s.so" % (k, prec))) for k in ("nl", "born"))

    def _g(self, g):
        # the double build is driven with the float-rounded values its getFloat reads
        return (g["nz"], g["nx"], float(np.float32(g["dz"])), float(np.float32(g["dx"])), g["nts"],
                float(np.float32(g["dts"])), g["S"], g["minPad"], float(np.float32(g["alphaCos"])))

    @staticmethod
    def wavefield_supported(g):
        """The reference's wavefield drivers size their device buffer with the
        32-bit product 5*nz*nx*nts; larger sizes are never run."""
        return 5 * int(g["nts"]) * int(g["nz"]) * int(g["nx"]) < 2 ** 31

    def nl_prop(self, adj, g, medium5, model5, data5, srcPos, recPos, wavefield=None):
        ns = (ctypes.c_int * 4)(*[len(p) for p in srcPos])
        nr = (ctypes.c_int * 4)(*[len(p) for p in recPos])
        sp = [np.ascontiguousarray(p, np.int32) for p in srcPos]
        rp = [np.ascontiguousarray(p, np.int32) for p in recPos]
        if wavefield is None:
            r = self.nl.ref_nl_prop(adj, *self._g(g), _pp(medium5, None), _pp(model5, None), _pp(data5, None),
                                    _pp(sp, None), ns, _pp(rp, None), nr, int(g.get("surface", 0)))
        else:
            if g.get("surface", 0):
                raise ValueError("the reference's wavefield drivers are driven here without the free surface")
            if not self.wavefield_supported(g):
                raise ValueError("reference wavefield drivers overflow their 32-bit buffer size at this size")
            assert wavefield.dtype == self.dt and wavefield.flags["C_CONTIGUOUS"]
            assert wavefield.shape == (g["nts"], 5, g["nx"], g["nz"])
            r = self.nl.ref_nl_prop_wf(adj, *self._g(g), _pp(medium5, None), _pp(model5, None), _pp(data5, None),
                                       _pp(sp, None), ns, _pp(rp, None), nr, wavefield.ctypes.data)
        assert r == 0

    @staticmethod
    def born_supported(g):
        """The reference's Born drivers index the coarse history with the 32-bit
        product its*nz*nx (kernelsGpuElastic.cu:1342) and fault once
        nts*nz*nx >= 2^31; those sizes are never run."""
        return int(g["nts"]) * int(g["nz"]) * int(g["nx"]) < 2 ** 31

    def born_prop(self, adj, g, medium5, srcDtw5, dm5, data5, srcPos, recPos):
        if not self.born_supported(g):
            raise ValueError("reference Born drivers overflow their 32-bit history index at this size")
        ns = (ctypes.c_int * 4)(*[len(p) for p in srcPos])
        nr = (ctypes.c_int * 4)(*[len(p) for p in recPos])
        sp = [np.ascontiguousarray(p, np.int32) for p in srcPos]
        rp = [np.ascontiguousarray(p, np.int32) for p in recPos]
        r = self.born.ref_born_prop(adj, *self._g(g), _pp(medium5, None), _pp(srcDtw5, None), _pp(dm5, None),
                                    _pp(data5, None), _pp(sp, None), ns, _pp(rp, None), nr)
        assert r == 0


# ====================================================================== operator level
class Case:
    """Everything the operator-level oracle needs, in plain arrays.

    ep [3][nx][nz]; par: dict of fdParamElastic keys; src: list (per shot) of
    (zc, xc) coordinate arrays; rec: (zc, xc) (constant geometry); grid
    origin oz, ox."""

    def __init__(self, ep, par, oz, ox, src, rec, method="linear", nfilt=1):
        self.ep = ep
        self.par = dict(par)
        self.oz, self.ox = float(oz), float(ox)
        self.src = src
        self.rec = rec
        self.method = method
        self.nfilt = nfilt

    @classmethod
    def from_workload(cls, w, method="linear", nfilt=1):
        src = [(w.src_z[e:e + 1], w.src_x[e:e + 1]) for e in range(w.nExp)]
        return cls(w.elastic.getNdArray(), w.par.as_dict(), w.oz, w.ox, src, (w.rec_z, w.rec_x), method, nfilt)

    def grid(self):
        p = self.par
        S = 2 * int(p["sub"])
        surface = int(p.get("surfaceCondition", 0))
        # fdParamElastic.cpp:43-44,74: with the free surface the top pad is not a taper
        zPad = int(p["zPadPlus"]) if surface else min(int(p["zPadMinus"]), int(p["zPadPlus"]))
        minPad = min(zPad, int(p["xPadMinus"]), int(p["xPadPlus"]))
        return dict(nz=int(p["nz"]), nx=int(p["nx"]), dz=float(p["dz"]), dx=float(p["dx"]), nts=int(p["nts"]),
                    dts=float(p["dts"]), S=S, minPad=minPad, alphaCos=float(p.get("alphaCos", 0.99)),
                    ots=float(p.get("ots", 0.0)), surface=surface)


def _stag_hypers(c):
    g = c.grid()
    dz, dx = np.float32(g["dz"]), np.float32(g["dx"])
    oz, ox = np.float32(c.oz), np.float32(c.ox)
    zs, xs = np.float32(oz - 0.5 * dz), np.float32(ox - 0.5 * dx)
    return [(oz, ox), (oz, xs), (zs, ox), (zs, xs)]   # center, x, z, xz


def _grids(orc, c, zc, xc):
    g = c.grid()
    return [orc.sinterp(zc, xc, g["nz"], o[0], g["dz"], g["nx"], o[1], g["dx"], c.method, c.nfilt)
            for o in _stag_hypers(c)]


def _scale_sources(orc, g, med, grids, reg, adjoint_order=False):
    """nonlinearPropElasticGpu.cpp:119-144 (forward order) / :425-452 (adjoint order)."""
    dt = orc.dt
    dtw = dt(np.float32(g["dts"])) / dt(g["S"])
    tdtw = dt(2.0) * dtw
    area = dt(np.float64(1.0) / np.float64(np.float32(g["dx"]) * np.float32(g["dz"])))

    def by_dtw():
        for f in range(5):
            G = grids[FIELD_GRID[f]]
            if f == 0:
                reg[f] *= med[0].ravel()[G["uniq"]][:, None]
            elif f == 1:
                reg[f] *= med[1].ravel()[G["uniq"]][:, None]
            else:
                reg[f] *= tdtw

    if adjoint_order:
        for f in range(5):
            reg[f] *= area
        by_dtw()
    else:
        by_dtw()
        for f in range(5):
            reg[f] *= area


def _reg_pos(grids):
    return [G["uniq"] for G in grids]


def scale_adjoint_wavefield(orc, g, med, W):
    """nonlinearPropElasticGpu.cpp:432-446: vx by rhoxDtw*area, vz by rhozDtw*area
    (products in the working precision), the stresses by 2*dtw*area in double."""
    dt = orc.dt
    dtw = dt(np.float32(g["dts"])) / dt(g["S"])
    area = dt(np.float64(1.0) / np.float64(np.float32(g["dx"]) * np.float32(g["dz"])))
    W[:, 0] *= (med[0] * area).astype(dt)
    W[:, 1] *= (med[1] * area).astype(dt)
    fac = np.float64(2.0) * np.float64(dtw) * np.float64(area)
    W[:, 2:] = (W[:, 2:].astype(np.float64) * fac).astype(dt)
    return W


def nl_forward(orc, c, model, engine=None, wshot=None):
    """model [nModelExp][5][nSrc][nts] -> data [nExp][5][nRec][nts] (add = False).
    wshot: shot index whose wavefield [nts][5][nx][nz] is saved and returned too."""
    g = c.grid()
    dt = orc.dt
    med = orc.medium(c.ep, g["dts"], g["S"])
    rec = _grids(orc, c, *c.rec)
    nrec = c.rec[0].size
    nts = g["nts"]
    data = np.zeros((len(c.src), 5, nrec, nts), dt)
    eng = engine or orc
    for e, (zc, xc) in enumerate(c.src):
        src = _grids(orc, c, zc, xc)
        m = np.ascontiguousarray(model[0 if model.shape[0] == 1 else e], dt)
        reg = []
        for f in range(5):
            G = src[FIELD_GRID[f]]
            r = np.zeros((len(G["uniq"]), nts), dt)
            orc.sinterp_apply(G, 1, 0, r, np.ascontiguousarray(m[f]))
            reg.append(r)
        _scale_sources(orc, g, med, src, reg)
        dreg = [np.zeros((len(rec[FIELD_GRID[f]]["uniq"]), nts), dt) for f in range(5)]
        if e == wshot:
            W = np.zeros((nts, 5, g["nx"], g["nz"]), dt)
            eng.nl_prop(0, g, med, reg, dreg, _reg_pos(src), _reg_pos(rec), W)
        else:
            eng.nl_prop(0, g, med, reg, dreg, _reg_pos(src), _reg_pos(rec))
        for f in range(5):
            out = np.zeros((nrec, nts), dt)
            orc.sinterp_apply(rec[FIELD_GRID[f]], 0, 1, dreg[f], out)
            data[e, f] += out
    return data if wshot is None else (data, W)


def nl_adjoint(orc, c, data, nModelExp=1, engine=None, wshot=None):
    """data [nExp][5][nRec][nts] -> model [nModelExp][5][nSrc][nts] (add = False).
    wshot: shot index whose (scaled) adjoint wavefield is saved and returned too."""
    g = c.grid()
    dt = orc.dt
    med = orc.medium(c.ep, g["dts"], g["S"])
    rec = _grids(orc, c, *c.rec)
    nts = g["nts"]
    nsrc = c.src[0][0].size
    model = np.zeros((nModelExp, 5, nsrc, nts), dt)
    stack = np.zeros((5, nsrc, nts), dt)
    eng = engine or orc
    for e, (zc, xc) in enumerate(c.src):
        src = _grids(orc, c, zc, xc)
        d = np.ascontiguousarray(data[e], dt)
        dreg = []
        for f in range(5):
            G = rec[FIELD_GRID[f]]
            r = np.zeros((len(G["uniq"]), nts), dt)
            orc.sinterp_apply(G, 1, 0, r, np.ascontiguousarray(d[f]))
            dreg.append(r)
        reg = [np.zeros((len(src[FIELD_GRID[f]]["uniq"]), nts), dt) for f in range(5)]
        if e == wshot:
            W = np.zeros((nts, 5, g["nx"], g["nz"]), dt)
            eng.nl_prop(1, g, med, reg, dreg, _reg_pos(src), _reg_pos(rec), W)
            scale_adjoint_wavefield(orc, g, med, W)
        else:
            eng.nl_prop(1, g, med, reg, dreg, _reg_pos(src), _reg_pos(rec))
        _scale_sources(orc, g, med, src, reg, adjoint_order=True)
        target = stack if nModelExp == 1 else np.zeros((5, nsrc, nts), dt)
        for f in range(5):
            orc.sinterp_apply(src[FIELD_GRID[f]], 0, 1, reg[f], target[f])
        if nModelExp != 1:
            model[e] += target
    if nModelExp == 1:
        model[0] += stack
    return model if wshot is None else (model, W)


def born_sources(orc, c, g, med, src, sig):
    dt = orc.dt
    nts = g["nts"]
    ntw = (nts - 1) * g["S"] + 1
    reg = []
    for f in range(5):
        G = src[FIELD_GRID[f]]
        r = np.zeros((len(G["uniq"]), nts), dt)
        orc.sinterp_apply(G, 1, 0, r, np.ascontiguousarray(sig[f], dt))
        reg.append(r)
    _scale_sources(orc, g, med, src, reg)
    fine = []
    for f in range(5):
        fn = np.zeros((reg[f].shape[0], ntw), dt)
        orc.tinterp(0, 0, nts, g["dts"], g.get("ots", 0.0), g["S"], reg[f], fn)
        fine.append(fn)
    return fine


def born_model_slice(orc, g, med, model):
    dt = orc.dt
    model = np.ascontiguousarray(model, dt)
    nx, nz = model.shape[1], model.shape[2]
    sl = [np.zeros((nx, nz), dt) for _ in range(5)]
    orc.stagger(0, 1, 0, sl[0], np.ascontiguousarray(model[0]))
    orc.stagger(1, 1, 0, sl[1], np.ascontiguousarray(model[0]))
    sl[2][...] = model[1]
    sl[3][...] = model[2]
    tmp = np.zeros((nx, nz), dt)
    orc.stagger(0, 1, 0, tmp, np.ascontiguousarray(model[2]))
    orc.stagger(1, 1, 0, sl[4], tmp)
    tdtw = np.float64(2.0) * np.float64(dt(np.float32(g["dts"])) / dt(g["S"]))
    sl[0] *= med[0]
    sl[1] *= med[1]
    for f in (2, 3, 4):
        sl[f][...] = (sl[f].astype(np.float64) * tdtw).astype(dt)
    return sl


def born_forward(orc, c, model, signals, engine=None):
    """model [3][nx][nz] -> data [nExp][5][nRec][nts] (add = False)."""
    g = c.grid()
    dt = orc.dt
    med = orc.medium(c.ep, g["dts"], g["S"])
    rec = _grids(orc, c, *c.rec)
    nrec = c.rec[0].size
    nts = g["nts"]
    sl = born_model_slice(orc, g, med, model)
    data = np.zeros((len(c.src), 5, nrec, nts), dt)
    eng = engine or orc
    for e, (zc, xc) in enumerate(c.src):
        src = _grids(orc, c, zc, xc)
        fine = born_sources(orc, c, g, med, src, signals[0 if len(signals) == 1 else e])
        dreg = [np.zeros((len(rec[FIELD_GRID[f]]["uniq"]), nts), dt) for f in range(5)]
        eng.born_prop(0, g, med, fine, [s.copy() for s in sl], dreg, _reg_pos(src), _reg_pos(rec))
        for f in range(5):
            out = np.zeros((nrec, nts), dt)
            orc.sinterp_apply(rec[FIELD_GRID[f]], 0, 1, dreg[f], out)
            data[e, f] += out
    return data


def born_adjoint(orc, c, data, signals, engine=None):
    """data [nExp][5][nRec][nts] -> model [3][nx][nz] (add = False)."""
    g = c.grid()
    dt = orc.dt
    med = orc.medium(c.ep, g["dts"], g["S"])
    rec = _grids(orc, c, *c.rec)
    nts = g["nts"]
    nx, nz = g["nx"], g["nz"]
    sl = [np.zeros((nx, nz), dt) for _ in range(5)]
    eng = engine or orc
    for e, (zc, xc) in enumerate(c.src):
        src = _grids(orc, c, zc, xc)
        fine = born_sources(orc, c, g, med, src, signals[0 if len(signals) == 1 else e])
        dreg = []
        for f in range(5):
            G = rec[FIELD_GRID[f]]
            r = np.zeros((len(G["uniq"]), nts), dt)
            orc.sinterp_apply(G, 1, 0, r, np.ascontiguousarray(data[e, f], dt))
            dreg.append(r)
        eng.born_prop(1, g, med, fine, sl, dreg, _reg_pos(src), _reg_pos(rec))
    tdtw = np.float64(2.0) * np.float64(dt(np.float32(g["dts"])) / dt(g["S"]))
    sl[0] *= med[0]
    sl[1] *= med[1]
    for f in (2, 3, 4):
        sl[f][...] = (sl[f].astype(np.float64) * tdtw).astype(dt)
    model = np.zeros((3, nx, nz), dt)
    t1 = model[0].copy()
    orc.stagger(0, 0, 1, sl[0], t1)
    orc.stagger(1, 0, 1, sl[1], t1)
    model[0] = t1
    t2 = np.zeros((nx, nz), dt)
    orc.stagger(1, 0, 0, sl[4], t2)
    t3 = np.zeros((nx, nz), dt)
    orc.stagger(0, 0, 0, t2, t3)
    model[1] += sl[2]
    model[2] += sl[3] + t3
    return model


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    den = np.linalg.norm(b.ravel())
    return float(np.linalg.norm((a - b).ravel()) / (den if den > 0 else 1.0))
