"""Operator classes of the elastic propagation path, drop-in for the reference's
pybind11 modules ``pyElastic_iso_float_nl`` / ``pyElastic_iso_float_born`` and
the Python wrappers of ``Elastic_iso_float_prop.py``.

Same class names, constructor arguments, method names, argument meaning and
``add`` semantics as the reference:

* ``spaceInterpGpu(zCoord, xCoord, gridHyper, nt, method, nFilt, dipole,
  zDipoleShift, xDipoleShift)``            (PF/pyElastic_iso_float_nl.cpp:19-30)
* ``nonlinearPropElasticShotsGpu(elasticParam, par, 8 geometry lists)`` with
  ``forward``, ``adjoint``, ``setBackground``, ``dotTest``
                                            (PF/pyElastic_iso_float_nl.cpp:32-54)
* ``BornElasticShotsGpu(elasticParam, par, sourcesSignalsVector, 8 geometry
  lists)`` with ``forward``, ``adjoint``, ``setBackground``, ``dotTest``
                                            (PF/pyElastic_iso_float_born.cpp:19-36)
* ``buildSourceGeometry`` / ``buildReceiversGeometry``
                                            (PF/Elastic_iso_float_prop.py:205-364, 525-661)

(PF = elastic_iso_lib/python/python_float of the reference project.)
Every numerical call goes through the CUDA library; errors from the C ABI
(QC failures, bounds, CUDA) surface as ``EioError``.
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import EioError, check, fptr, iptr
from .sepvec import axis, hypercube, floatVector, getSepVector, paramObj

__all__ = [
    "EioError", "spaceInterpGpu", "nonlinearPropElasticShotsGpu", "BornElasticShotsGpu",
    "buildSourceGeometry", "buildReceiversGeometry", "fd_params_from_par",
]

_FIELD_GRID = (1, 2, 0, 0, 3)   # vx -> x grid, vz -> z grid, sxx/szz -> center, sxz -> xz


def _arr(v, dtype=np.float32):
    a = v.getNdArray() if hasattr(v, "getNdArray") else np.asarray(v)
    return np.ascontiguousarray(a, dtype=dtype)


def _hyper_of(v):
    return v.getHyper() if hasattr(v, "getHyper") else None


class spaceInterpGpu:
    """Irregular acquisition devices <-> unique regular grid points
    (spaceInterpGpu, F/src/spaceInterpGpu.cpp:11-362)."""

    def __init__(self, zCoord, xCoord, gridHyper, nt, method="linear", nFilt=1, dipole=0,
                 zDipoleShift=0.0, xDipoleShift=0.0):
        z = _arr(zCoord).ravel()
        x = _arr(xCoord).ravel()
        if z.size != x.size:
            raise ValueError("zCoord and xCoord must have the same length")
        az, ax = gridHyper.getAxis(1), gridHyper.getAxis(2)
        L = _lib.lib()
        h = ctypes.c_void_p()
        check(L.eio_sinterp_create(fptr(z), fptr(x), int(z.size), az.n, az.o, az.d, ax.n, ax.o, ax.d, int(nt),
                                   method.encode(), int(nFilt), int(dipole), float(zDipoleShift),
                                   float(xDipoleShift), ctypes.byref(h)))
        self._h = h
        self._L = L
        self.nt = int(nt)
        self.gridHyper = gridHyper
        self.zCoord, self.xCoord = z.copy(), x.copy()   # the irregular device coordinates
        self.method, self.nFilt = method, int(nFilt)
        ni, nr, nf = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        check(L.eio_sinterp_sizes(h, ctypes.byref(ni), ctypes.byref(nr), ctypes.byref(nf)))
        self.nDeviceIrreg, self.nDeviceReg, self.nFiltTotal = ni.value, nr.value, nf.value
        pos = np.zeros(max(self.nDeviceReg, 1), dtype=np.int32)
        check(L.eio_sinterp_positions(h, iptr(pos)))
        self.regPosUnique = pos[: self.nDeviceReg].copy()

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self._L.eio_sinterp_destroy(h)
            self._h = None

    @property
    def handle(self):
        return self._h

    def getNDeviceReg(self):
        return self.nDeviceReg

    def getNDeviceIrreg(self):
        return self.nDeviceIrreg

    def getRegPosUnique(self):
        return self.regPosUnique

    def getWeights(self):
        n = self.nDeviceIrreg * self.nFiltTotal
        gpi = np.zeros(max(n, 1), dtype=np.int32)
        w = np.zeros(max(n, 1), dtype=np.float32)
        check(self._L.eio_sinterp_weights(self._h, iptr(gpi), fptr(w)))
        return gpi[:n], w[:n]

    def getInfo(self):
        gpi, w = self.getWeights()
        lines = ["---------- Space Interp Info ----------",
                 "_nDeviceIrreg= %d" % self.nDeviceIrreg, "_nDeviceRreg= %d" % self.nDeviceReg]
        for i in range(self.nDeviceIrreg):
            lines.append("Irreg Device %d weights %s" % (i, w[i * self.nFiltTotal:(i + 1) * self.nFiltTotal]))
        return "\n".join(lines)

    def forward(self, add, signalReg, signalIrreg):
        """regular [nReg][nt] -> irregular [nIrreg][nt]"""
        reg = _arr(signalReg)
        out = signalIrreg.getNdArray() if hasattr(signalIrreg, "getNdArray") else signalIrreg
        res = np.ascontiguousarray(out, dtype=np.float32)
        check(self._L.eio_sinterp_forward(self._h, int(bool(add)), fptr(reg), fptr(res)))
        if res is not out:
            out[...] = res
        return out

    def adjoint(self, add, signalReg, signalIrreg):
        irr = _arr(signalIrreg)
        out = signalReg.getNdArray() if hasattr(signalReg, "getNdArray") else signalReg
        res = np.ascontiguousarray(out, dtype=np.float32)
        check(self._L.eio_sinterp_adjoint(self._h, int(bool(add)), fptr(res), fptr(irr)))
        if res is not out:
            out[...] = res
        return out


def fd_params_from_par(par, elasticParam):
    """eio_fd_params from a paramObj (keys of fdParamElastic.cpp:18-77) and the
    elastic-parameter vector (whose first two axes give oz, ox)."""
    if isinstance(par, dict):
        par = paramObj(par)
    p = _lib.FdParams()
    _lib.lib().eio_fd_params_default(ctypes.byref(p))
    hyp = _hyper_of(elasticParam)
    p.nts = par.getInt("nts")
    p.dts = par.getFloat("dts", 0.0)
    p.ots = par.getFloat("ots", 0.0)
    p.sub = par.getInt("sub")
    p.nz = par.getInt("nz")
    p.nx = par.getInt("nx")
    p.dz = par.getFloat("dz", -1.0)
    p.dx = par.getFloat("dx", -1.0)
    p.oz = hyp.getAxis(1).o if hyp is not None else par.getFloat("oz", 0.0)
    p.ox = hyp.getAxis(2).o if hyp is not None else par.getFloat("ox", 0.0)
    p.zPadMinus = par.getInt("zPadMinus")
    p.zPadPlus = par.getInt("zPadPlus")
    p.xPadMinus = par.getInt("xPadMinus")
    p.xPadPlus = par.getInt("xPadPlus")
    p.fMax = par.getFloat("fMax", 1000.0)
    p.blockSize = par.getInt("blockSize", 16)
    p.fat = par.getInt("fat", 4)
    p.alphaCos = par.getFloat("alphaCos", 0.99)
    p.surfaceCondition = par.getInt("surfaceCondition", 0)
    p.mod_par = par.getInt("mod_par", 1)
    p.errorTolerance = par.getFloat("errorTolerance", 0.000001)
    if hyp is not None:
        # checkParfileConsistencySpace, F/src/fdParamElastic.cpp:308-326
        scale = 1000.0 if p.mod_par == 2 else 1.0
        tol = p.errorTolerance
        az, ax = hyp.getAxis(1), hyp.getAxis(2)
        dz = p.dz * (1000.0 if p.mod_par == 2 else 1.0)
        dx = p.dx * (1000.0 if p.mod_par == 2 else 1.0)
        if p.nz != az.n or abs(dz - az.d * scale) > tol:
            raise EioError(-2, "**** ERROR: nz/dz not consistent with parfile ****")
        if p.nx != ax.n or abs(dx - ax.d * scale) > tol:
            raise EioError(-2, "**** ERROR: nx/dx not consistent with parfile ****")
    return p


def _device_from_par(par):
    ids = par.getInts("iGpu", [-1])
    if ids and ids[0] >= 0:
        return int(ids[0])
    return 0


class _ElasticOp:
    """Shared state of the two multi-shot operators: one device context
    (fdParamElastic + device allocation) on the first GPU of the list."""

    def __init__(self, elasticParam, par, src, rec):
        if isinstance(par, dict):
            par = paramObj(par)
        self.par = par
        self.nExp = par.getInt("nExp")
        self.fd = fd_params_from_par(par, elasticParam)
        self.device = _device_from_par(par)
        ep = _arr(elasticParam)
        if ep.size != 3 * self.fd.nz * self.fd.nx:
            raise EioError(-1, "elastic parameter size does not match nz*nx*3")
        self._L = _lib.lib()
        h = ctypes.c_void_p()
        check(self._L.eio_ctx_create(ctypes.byref(self.fd), fptr(ep), self.device, ctypes.byref(h)))
        self._ctx = h
        self.src = [list(g) for g in src]
        self.rec = [list(g) for g in rec]
        if any(len(g) != self.nExp for g in self.src):
            raise EioError(-1, "each source geometry list must hold nExp interpolators")
        nrg = {len(g) for g in self.rec}
        if len(nrg) != 1 or list(nrg)[0] not in (1, self.nExp):
            raise EioError(-1, "receiver geometry lists must hold 1 or nExp interpolators")
        self.nRecGeom = len(self.rec[0])
        self._src_arr = _lib.ptr_array([g[i].handle.value for i in range(self.nExp) for g in self.src])
        self._rec_arr = _lib.ptr_array([g[i].handle.value for i in range(self.nRecGeom) for g in self.rec])
        self.nSrcIrreg = self.src[0][0].nDeviceIrreg
        self.nRecIrreg = self.rec[0][0].nDeviceIrreg

    def __del__(self):
        h = getattr(self, "_ctx", None)
        if h is not None and h.value:
            self._L.eio_ctx_destroy(h)
            self._ctx = None

    @property
    def ctx(self):
        return self._ctx

    # ---- cropped shots (no reference counterpart)
    def setShotWindows(self, ix0, nxw):
        """Propagate shot i on grid columns [ix0[i], ix0[i] + nxw[i]) only
        (eio_ctx_set_shot_windows): a window holds 2*fat + a multiple of 16
        columns and the shot's devices in its updated interior, and the grid's
        cosine taper runs from its edges."""
        ix0 = np.ascontiguousarray(ix0, dtype=np.int32)
        nxw = np.ascontiguousarray(nxw, dtype=np.int32)
        if ix0.shape != (self.nExp,) or nxw.shape != (self.nExp,):
            raise EioError(-1, "one window per shot (nExp = %d)" % self.nExp)
        check(self._L.eio_ctx_set_shot_windows(self._ctx, self.nExp, _lib.iptr(ix0), _lib.iptr(nxw)))
        self.shotWindows = (ix0, nxw)

    def clearShotWindows(self):
        check(self._L.eio_ctx_set_shot_windows(self._ctx, 0, None, None))
        self.shotWindows = None

    def autoShotWindows(self, margin=None):
        """Set per-shot windows spanning each shot's sources and receivers plus
        ``margin`` columns on both sides (default: the grid's wider x pad), plus
        the fat frame, widened to 2*fat + a multiple of 16 columns and kept in
        the grid.  Returns (ix0, nxw)."""
        nz, nx, fat = self.fd.nz, self.fd.nx, self.fd.fat
        if margin is None:
            margin = max(self.fd.xPadMinus, self.fd.xPadPlus)
        ix0s, nxws = [], []
        for e in range(self.nExp):
            cols = []
            for g in self.src:
                cols.append(np.asarray(g[e].getRegPosUnique()) // nz)
            for g in self.rec:
                cols.append(np.asarray(g[0 if self.nRecGeom == 1 else e].getRegPosUnique()) // nz)
            cols = np.concatenate([c for c in cols if c.size])
            lo = max(int(cols.min()) - margin - fat, 0)
            hi = min(int(cols.max()) + margin + fat + 1, nx)
            w = hi - lo
            w = 2 * fat + 16 * int(np.ceil(max(w - 2 * fat, 16) / 16.0))
            w = min(w, nx)
            lo = min(max(lo - (w - (hi - lo)) // 2, 0), nx - w)
            ix0s.append(lo)
            nxws.append(w)
        self.setShotWindows(ix0s, nxws)
        return np.array(ix0s, np.int32), np.array(nxws, np.int32)

    def setBackground(self, elasticParam):
        """Rebuild the medium (fdParamElastic QC runs again and may raise)."""
        ep = _arr(elasticParam)
        check(self._L.eio_ctx_set_background(self._ctx, fptr(ep)))

    def setCheckpointPrecision(self, mode):
        """Born source-wavefield snapshots: 0 FP32, 1 BF16, 2 FP16."""
        check(self._L.eio_ctx_set_checkpoint_precision(self._ctx, int(mode)))

    def setLanes(self, lanes):
        """Shots of one multi-shot call run on up to ``lanes`` engines of this
        context (default 2), each on its own stream and host thread."""
        check(self._L.eio_ctx_set_lanes(self._ctx, int(lanes)))

    def setShotBatch(self, shots):
        """Nonlinear operators: advance up to ``shots`` (1 .. 8, default 8) shots
        in lockstep with one step launch for all of them; 1 runs the shots one
        at a time on the lanes."""
        check(self._L.eio_ctx_set_shot_batch(self._ctx, int(shots)))

    def setBornBatch(self, shots):
        """Born operators: run the shots in lockstep groups of up to ``shots``
        (1 .. 8, capped by the lanes and the device memory); default 1, the
        shots one at a time on the lanes."""
        check(self._L.eio_ctx_set_born_batch(self._ctx, int(shots)))

    def setPersistent(self, mask):
        """Shot groups of the Born operators: the propagation phases that run
        every fine step in one persistent launch (bits: 1 source wavefield, 2
        scattered wavefield, 4 adjoint; True = 7, False = 0 = one launch per step)."""
        mask = 7 if mask is True else 0 if mask is False else int(mask)
        check(self._L.eio_ctx_set_persistent(self._ctx, mask))

    def getMedium(self):
        n = self.fd.nz * self.fd.nx
        out = [np.zeros((self.fd.nx, self.fd.nz), np.float32) for _ in range(5)]
        check(self._L.eio_ctx_get_medium(self._ctx, *[fptr(o) for o in out]))
        return out

    def _check_time(self, vec):
        hyp = _hyper_of(vec)
        if hyp is None:
            return
        t = hyp.getAxis(1)
        tol = self.fd.errorTolerance
        if t.n != self.fd.nts or abs(t.d - self.fd.dts) > tol or abs(t.o - self.fd.ots) > tol:
            raise EioError(-2, "**** ERROR: nts/dts/ots not consistent with parfile ****")

    def _dot_test(self, model_space, data_space, verbose, maxError):
        """operator.h:50-89 dot-product test, with FP64 dot products."""
        d1 = model_space.clone().rand(1234)
        r1 = data_space.clone().rand(4321)
        d2 = model_space.clone()
        r2 = data_space.clone()
        from .fwi import dot64   # FP64 sums on the GPU
        self.forward(False, d1, r2)
        self.adjoint(False, d2, r1)
        dot1, dot2 = dot64(r1, r2), dot64(d1, d2)
        err_no_add = abs((dot1 - dot2) / dot2)
        self.forward(True, d1, r2)
        self.adjoint(True, d2, r1)
        dot3, dot4 = dot64(r1, r2), dot64(d1, d2)
        err_add = abs((dot3 - dot4) / dot4)
        if verbose:
            print("WITHOUT ADD:\ndot1: %.16g\ndot2: %.16g\nerror WITHOUT ADD: %.16g" % (dot1, dot2, err_no_add))
            print("WITH ADD:\ndot3: %.16g\ndot4: %.16g\nerror with ADD: %.16g" % (dot3, dot4, err_add))
        self.lastDotTest = (err_no_add, err_add)
        return err_no_add <= maxError and err_add <= maxError


class nonlinearPropElasticShotsGpu(_ElasticOp):
    """Nonlinear elastic propagation over many shots
    (nonlinearPropElasticShotsGpu, F/src/nonlinearPropElasticShotsGpu.cpp).

    model: [nts, nSrc, 5, nModelExp] (numpy (nModelExp, 5, nSrc, nts));
    data:  [nts, nRec, 5, nExp]      (numpy (nExp, 5, nRec, nts)).
    """

    def __init__(self, elasticParam, par, sourcesVectorCenterGrid, sourcesVectorXGrid, sourcesVectorZGrid,
                 sourcesVectorXZGrid, receiversVectorCenterGrid, receiversVectorXGrid, receiversVectorZGrid,
                 receiversVectorXZGrid):
        super().__init__(elasticParam, par,
                         [sourcesVectorCenterGrid, sourcesVectorXGrid, sourcesVectorZGrid, sourcesVectorXZGrid],
                         [receiversVectorCenterGrid, receiversVectorXGrid, receiversVectorZGrid,
                          receiversVectorXZGrid])

    def _shapes(self, model, data):
        m = model.getNdArray() if hasattr(model, "getNdArray") else model
        d = data.getNdArray() if hasattr(data, "getNdArray") else data
        if m.ndim == 3:
            m = m.reshape((1,) + m.shape)
        if m.shape[1] != 5:
            raise EioError(-1, "model must have five wavefield components")
        nme = m.shape[0]
        if m.shape[2:] != (self.nSrcIrreg, self.fd.nts) or d.shape != (self.nExp, 5, self.nRecIrreg, self.fd.nts):
            raise EioError(-1, "model/data shapes do not match the acquisition geometry")
        return m, d, nme

    def forward(self, add, model, data):
        self._check_time(model)
        self._check_time(data)
        m, d, nme = self._shapes(model, data)
        mm = np.ascontiguousarray(m, dtype=np.float32)
        dd = np.ascontiguousarray(d, dtype=np.float32)
        check(self._L.eio_nl_forward(self._ctx, int(bool(add)), self.nExp, nme, fptr(mm), fptr(dd),
                                     self._src_arr, self._rec_arr, self.nRecGeom))
        if dd is not d:
            d[...] = dd

    def adjoint(self, add, model, data):
        self._check_time(model)
        self._check_time(data)
        m, d, nme = self._shapes(model, data)
        mm = np.ascontiguousarray(m, dtype=np.float32)
        dd = np.ascontiguousarray(d, dtype=np.float32)
        check(self._L.eio_nl_adjoint(self._ctx, int(bool(add)), self.nExp, nme, fptr(mm), fptr(dd),
                                     self._src_arr, self._rec_arr, self.nRecGeom))
        if mm is not m:
            m[...] = mm

    # ---- wavefield output (nonlinearPropElasticShotsGpu.cpp:185-300, 424-540):
    # with par saveWavefield = 1 the shot wavefieldShotNumber (0-based) keeps its
    # wavefield [nts][5][nx][nz]; the adjoint one is scaled like the adjoint sources.
    def _wavefield_shot(self):
        save = self.par.getInt("saveWavefield", 0)
        shot = self.par.getInt("wavefieldShotNumber", 0)
        return shot if save != 0 and 0 <= shot < self.nExp else -1

    def _new_wavefield(self, shot):
        if shot < 0:
            return np.zeros((1, 1, 1, 1), np.float32)
        return np.zeros((self.fd.nts, 5, self.fd.nx, self.fd.nz), np.float32)

    def forwardWavefield(self, add, model, data):
        self._check_time(model)
        self._check_time(data)
        m, d, nme = self._shapes(model, data)
        mm = np.ascontiguousarray(m, dtype=np.float32)
        dd = np.ascontiguousarray(d, dtype=np.float32)
        shot = self._wavefield_shot()
        w = self._new_wavefield(shot)
        check(self._L.eio_nl_forward_wavefield(self._ctx, int(bool(add)), self.nExp, nme, fptr(mm), fptr(dd),
                                               self._src_arr, self._rec_arr, self.nRecGeom, shot, fptr(w)))
        if dd is not d:
            d[...] = dd
        self._wavefield = w

    def adjointWavefield(self, add, model, data):
        self._check_time(model)
        self._check_time(data)
        m, d, nme = self._shapes(model, data)
        mm = np.ascontiguousarray(m, dtype=np.float32)
        dd = np.ascontiguousarray(d, dtype=np.float32)
        shot = self._wavefield_shot()
        w = self._new_wavefield(shot)
        check(self._L.eio_nl_adjoint_wavefield(self._ctx, int(bool(add)), self.nExp, nme, fptr(mm), fptr(dd),
                                               self._src_arr, self._rec_arr, self.nRecGeom, shot, fptr(w)))
        if mm is not m:
            m[...] = mm
        self._wavefield = w

    def getWavefield(self):
        """The wavefield kept by the last forwardWavefield / adjointWavefield call
        (axes z, x, component, coarse time; numpy shape (nts, 5, nx, nz))."""
        w = getattr(self, "_wavefield", None)
        if w is None:
            w = self._new_wavefield(-1)
        if w.shape[0] == 1:
            return floatVector(hypercube(ns=[1, 1, 1, 1]), w.copy())
        t = axis(self.fd.nts, self.fd.ots, self.fd.dts)
        hz = axis(self.fd.nz, self.fd.oz, self.fd.dz)
        hx = axis(self.fd.nx, self.fd.ox, self.fd.dx)
        return floatVector(hypercube(axes=[hz, hx, axis(5), t]), w.copy())

    def prepareShot(self, iExp, model):
        """Regular-grid inputs of shot iExp for the single-shot eio_nl_fwd_reg_dev
        entry point: the irregular source traces ``model`` [5][nSrc][nts] spread and
        scaled onto the regular grid (5 arrays [nSrcReg(grid)][nts]) and the source /
        receiver position lists (grid order center, x, z, xz)."""
        src = [g[iExp] for g in self.src]
        rec = [g[0 if self.nRecGeom == 1 else iExp] for g in self.rec]
        m = np.ascontiguousarray(_arr(model).reshape(5, self.nSrcIrreg, self.fd.nts))
        reg = [np.zeros((src[_FIELD_GRID[f]].nDeviceReg, self.fd.nts), np.float32) for f in range(5)]
        check(self._L.eio_nl_prepare_sources(self._ctx, fptr(m), _lib.ptr_array([g.handle.value for g in src]),
                                             _lib.ptr_array([a.ctypes.data for a in reg])))
        return reg, [g.getRegPosUnique() for g in src], [g.getRegPosUnique() for g in rec]

    def modelSpace(self, nModelExp=1):
        t = axis(self.fd.nts, self.fd.ots, self.fd.dts)
        return floatVector(hypercube(axes=[t, axis(self.nSrcIrreg), axis(5), axis(nModelExp)]))

    def dataSpace(self):
        t = axis(self.fd.nts, self.fd.ots, self.fd.dts)
        return floatVector(hypercube(axes=[t, axis(self.nRecIrreg), axis(5), axis(self.nExp)]))

    def dotTest(self, verbose=False, maxError=0.00001):
        return self._dot_test(self.modelSpace(), self.dataSpace(), verbose, maxError)


class nonlinearFwiPropElasticShotsGpu(nonlinearPropElasticShotsGpu):
    """Nonlinear modelling as a function of the elastic parameters, for FWI
    (nonlinearFwiPropElasticShotsGpu, PF/Elastic_iso_float_prop.py:1107-1149):
    forward(add, model, data) sets model [3][nx][nz] as the background and
    propagates the fixed source signals ``sources`` [nts, nSrc, 5, 1].
    It has no adjoint (the reference wrapper defines none either)."""

    def __init__(self, elasticParam, par, sources, sourcesVectorCenterGrid, sourcesVectorXGrid,
                 sourcesVectorZGrid, sourcesVectorXZGrid, receiversVectorCenterGrid, receiversVectorXGrid,
                 receiversVectorZGrid, receiversVectorXZGrid):
        super().__init__(elasticParam, par, sourcesVectorCenterGrid, sourcesVectorXGrid, sourcesVectorZGrid,
                         sourcesVectorXZGrid, receiversVectorCenterGrid, receiversVectorXGrid, receiversVectorZGrid,
                         receiversVectorXZGrid)
        src = sources.getNdArray() if hasattr(sources, "getNdArray") else sources
        self.sources = np.array(src, dtype=np.float32, copy=True)

    def forward(self, add, model, data):
        self.setBackground(model)
        super().forward(add, self.sources, data)

    def adjoint(self, add, model, data):
        raise NotImplementedError("the nonlinear FWI operator has no adjoint; use BornElasticShotsGpu")


class BornElasticShotsGpu(_ElasticOp):
    """Born (linearised) elastic operator over (drho, dlambda, dmu)
    (BornElasticShotsGpu, F/src/BornElasticShotsGpu.cpp).

    model: [nz, nx, 3] (numpy (3, nx, nz)); data: [nts, nRec, 5, nExp];
    sourcesSignalsVector: list (1 or nExp) of [nts, nSrc, 5] vectors.
    """

    def __init__(self, elasticParam, par, sourcesSignalsVector, sourcesVectorCenterGrid, sourcesVectorXGrid,
                 sourcesVectorZGrid, sourcesVectorXZGrid, receiversVectorCenterGrid, receiversVectorXGrid,
                 receiversVectorZGrid, receiversVectorXZGrid):
        super().__init__(elasticParam, par,
                         [sourcesVectorCenterGrid, sourcesVectorXGrid, sourcesVectorZGrid, sourcesVectorXZGrid],
                         [receiversVectorCenterGrid, receiversVectorXGrid, receiversVectorZGrid,
                          receiversVectorXZGrid])
        self.elasticHyper = _hyper_of(elasticParam)
        self.setSourceSignals(sourcesSignalsVector)

    def setSourceSignals(self, sourcesSignalsVector):
        """Replace the source signals (1 or nExp of [nts, nSrc, 5]), e.g. by
        band-limited ones between the bands of a multiscale inversion.  The
        reference fixes them at construction; this is an extension."""
        sigs = []
        for s in sourcesSignalsVector:
            self._check_time(s)
            a = _arr(s).reshape(5, self.nSrcIrreg, self.fd.nts)
            sigs.append(np.ascontiguousarray(a, dtype=np.float32))
        if len(sigs) not in (1, self.nExp):
            raise EioError(-1, "sourcesSignalsVector must hold 1 or nExp signals")
        self._sigs = sigs
        self._sig_arr = _lib.ptr_array([a.ctypes.data for a in self._sigs])

    def _shapes(self, model, data):
        m = model.getNdArray() if hasattr(model, "getNdArray") else model
        d = data.getNdArray() if hasattr(data, "getNdArray") else data
        if m.shape != (3, self.fd.nx, self.fd.nz) or d.shape != (self.nExp, 5, self.nRecIrreg, self.fd.nts):
            raise EioError(-1, "model/data shapes do not match the grid or acquisition")
        return m, d

    def forward(self, add, model, data):
        self._check_time(data)
        m, d = self._shapes(model, data)
        mm = np.ascontiguousarray(m, dtype=np.float32)
        dd = np.ascontiguousarray(d, dtype=np.float32)
        check(self._L.eio_born_forward(self._ctx, int(bool(add)), self.nExp, fptr(mm), fptr(dd), self._sig_arr,
                                       len(self._sigs), self._src_arr, self._rec_arr, self.nRecGeom))
        if dd is not d:
            d[...] = dd

    def adjoint(self, add, model, data):
        self._check_time(data)
        m, d = self._shapes(model, data)
        mm = np.ascontiguousarray(m, dtype=np.float32)
        dd = np.ascontiguousarray(d, dtype=np.float32)
        check(self._L.eio_born_adjoint(self._ctx, int(bool(add)), self.nExp, fptr(mm), fptr(dd), self._sig_arr,
                                       len(self._sigs), self._src_arr, self._rec_arr, self.nRecGeom))
        if mm is not m:
            m[...] = mm

    _COMP_CODES = {"vx": 0, "vz": 1, "sxx": 2, "szz": 3, "sxz": 4, "p": 5}

    def fwiGradient(self, elasticModel, sources, dObs, components=None, data=None):
        """Misfit and gradient of 0.5 ||S F(m) - dObs||^2 in one pass per shot.

        Sets elasticModel [3][nx][nz] as the background, then per shot runs the
        nonlinear forward of ``sources`` (the source traces of
        nonlinearFwiPropElasticShotsGpu, [nModelExp][5][nSrc][nts], nModelExp 1
        or nExp) while recording the Born source wavefield, forms the residual
        of the sampled components and runs the Born adjoint on the recorded
        wavefield (two propagations per shot; the reference runs the nonlinear
        forward, then BornElasticShotsGpu's adjoint, which propagates the source
        again).  ``components``: a comma-separated list of vx, vz, sxx, szz, sxz,
        p (ElasticDatComp's), all five fields when None; dObs has the sampled
        shape [nExp][nComp][nRec][nts].  ``data`` (optional, [nExp][5][nRec][nts])
        receives the modelled data.  Returns (misfit, gradient [3][nx][nz]).
        No free surface (the Born operator has none)."""
        comps = ["vx", "vz", "sxx", "szz", "sxz"] if components is None else \
            [c.strip().lower() for c in components.split(",")]
        if len(set(comps)) != len(comps) or any(c not in self._COMP_CODES for c in comps):
            raise EioError(-1, "unknown or repeated data component in %r" % (components,))
        codes = np.array([self._COMP_CODES[c] for c in comps], np.int32)
        self.setBackground(elasticModel)
        src = np.ascontiguousarray(_arr(sources), dtype=np.float32)
        per = 5 * self.nSrcIrreg * self.fd.nts
        if src.size % per or src.size // per not in (1, self.nExp):
            raise EioError(-1, "sources must hold 1 or nExp shots of [5][nSrc][nts] traces")
        d_obs = np.ascontiguousarray(_arr(dObs), dtype=np.float32)
        if d_obs.shape != (self.nExp, len(comps), self.nRecIrreg, self.fd.nts):
            raise EioError(-1, "dObs shape %s, expected %s" % (d_obs.shape, (self.nExp, len(comps),
                                                                               self.nRecIrreg, self.fd.nts)))
        dd = None
        if data is not None:
            dd = _arr(data)
            if dd.shape != (self.nExp, 5, self.nRecIrreg, self.fd.nts) or not dd.flags["C_CONTIGUOUS"]:
                raise EioError(-1, "data must be a contiguous float32 [nExp][5][nRec][nts] array")
        grad = np.zeros((3, self.fd.nx, self.fd.nz), np.float32)
        phi = ctypes.c_double()
        check(self._L.eio_fwi_gradient(self._ctx, self.nExp, src.size // per, fptr(src), fptr(d_obs), len(codes),
                                       _lib.iptr(codes), self._src_arr, self._rec_arr, self.nRecGeom,
                                       None if dd is None else dd.ctypes.data, fptr(grad), ctypes.byref(phi)))
        return phi.value, grad

    def prepareShot(self, iExp):
        """Regular-grid inputs of shot iExp for the single-shot *_reg_dev entry
        points: 5 scaled fine-time source traces and the source / receiver
        position lists (grid order center, x, z, xz)."""
        src = [g[iExp] for g in self.src]
        rec = [g[0 if self.nRecGeom == 1 else iExp] for g in self.rec]
        ntw = (self.fd.nts - 1) * 2 * self.fd.sub + 1
        fine = [np.zeros((src[_FIELD_GRID[f]].nDeviceReg, ntw), np.float32) for f in range(5)]
        sig = self._sigs[0 if len(self._sigs) == 1 else iExp]
        check(self._L.eio_born_prepare_sources(self._ctx, fptr(sig), _lib.ptr_array([g.handle.value for g in src]),
                                               _lib.ptr_array([a.ctypes.data for a in fine])))
        return fine, [g.getRegPosUnique() for g in src], [g.getRegPosUnique() for g in rec]

    def prepareModel(self, model):
        """(drho, dlambda, dmu) [3][nx][nz] -> the 5 staggered, scaled perturbation grids."""
        m = _arr(model).reshape(3, self.fd.nx, self.fd.nz)
        out = [np.zeros((self.fd.nx, self.fd.nz), np.float32) for _ in range(5)]
        check(self._L.eio_born_prepare_model(self._ctx, fptr(m), _lib.ptr_array([a.ctypes.data for a in out])))
        return out

    def modelSpace(self):
        if self.elasticHyper is not None:
            return floatVector(self.elasticHyper.clone())
        return floatVector(hypercube(ns=[self.fd.nz, self.fd.nx, 3]))

    def dataSpace(self):
        t = axis(self.fd.nts, self.fd.ots, self.fd.dts)
        return floatVector(hypercube(axes=[t, axis(self.nRecIrreg), axis(5), axis(self.nExp)]))

    def dotTest(self, verbose=False, maxError=0.00001):
        return self._dot_test(self.modelSpace(), self.dataSpace(), verbose, maxError)


# ---------------------------------------------------------------------------
# Acquisition geometry builders, PF/Elastic_iso_float_prop.py:205-364, 525-661
# ---------------------------------------------------------------------------
def _staggered_hypers(elasticParam):
    h = elasticParam.getHyper()
    az, ax = h.getAxis(1), h.getAxis(2)
    pax = h.getAxis(3) if h.getNdim() >= 3 else axis(3)
    z = axis(az.n, az.o, az.d)
    zs = axis(az.n, az.o - 0.5 * az.d, az.d)
    x = axis(ax.n, ax.o, ax.d)
    xs = axis(ax.n, ax.o - 0.5 * ax.d, ax.d)
    return (hypercube(axes=[z, x, pax]), hypercube(axes=[z, xs, pax]),
            hypercube(axes=[zs, x, pax]), hypercube(axes=[zs, xs, pax]))


def _four_grids(zc, xc, hypers, nts, method, nfilt, dipole, zds, xds):
    return [spaceInterpGpu(zc, xc, h, nts, method, nfilt, dipole, zds, xds) for h in hypers]


def _geometry_array(geom):
    """A geometry file's coordinates [3][nPoints][nExp] (numpy order; x, y, z
    along the slowest axis): a SEP dataset read with ndims = 3, as the
    reference reads it (genericIO.defaultIO.getVector(file, ndims=3),
    python_float/Elastic_iso_float_prop.py:269-270), a ``.npy`` array, or an
    array given directly."""
    if isinstance(geom, str):
        if geom.endswith(".npy"):
            return np.load(geom)
        from .sepio import readSep
        return np.asarray(readSep(geom, ndims=3).getNdArray())
    return np.asarray(geom)


def buildSourceGeometry(parObject, elasticParam):
    """Sources on the four staggered grids, one set per shot.
    Returns (center, x, z, xz) lists and the shot axis."""
    if isinstance(parObject, dict):
        parObject = paramObj(parObject)
    dipole = parObject.getInt("dipole", 0)
    zds = parObject.getFloat("zDipoleShift", 0.0)
    xds = parObject.getFloat("xDipoleShift", 0.0)
    nts = parObject.getInt("nts")
    nExp = parObject.getInt("nExp")
    h = elasticParam.getHyper()
    dz, oz = h.getAxis(1).d, h.getAxis(1).o
    dx, ox = h.getAxis(2).d, h.getAxis(2).o
    hypers = _staggered_hypers(elasticParam)
    method = parObject.getString("sourceInterpMethod", "linear")
    nfilt = parObject.getInt("sourceInterpNumFilters", 4)
    lists = ([], [], [], [])
    geom = parObject.getString("sourceGeomFile", "None")
    if geom != "None":
        # numpy array [3][nSimSou][nExp] (x, y, z coordinates), as read from the geometry file
        g = _geometry_array(geom)
        if g.shape[2] != nExp:
            raise ValueError("ERROR! nExp (%d) not consistent with number of shots provided within "
                             "sourceGeomFile (%d)" % (nExp, g.shape[2]))
        sourceAxis = axis(nExp, 1.0, 1.0)
        for iExp in range(nExp):
            zc = np.ascontiguousarray(g[2, :, iExp], dtype=np.float32)
            xc = np.ascontiguousarray(g[0, :, iExp], dtype=np.float32)
            for lst, grid in zip(lists, _four_grids(zc, xc, hypers, nts, method, nfilt, dipole, zds, xds)):
                lst.append(grid)
    else:
        ozs = parObject.getInt("zSource") - 1 + parObject.getInt("zPadMinus") + parObject.getInt("fat", 4)
        oxs = parObject.getInt("xSource") - 1 + parObject.getInt("xPadMinus") + parObject.getInt("fat", 4)
        spacing = parObject.getInt("spacingShots")
        sourceAxis = axis(nExp, ox + oxs * dx, spacing * dx)
        for iExp in range(nExp):
            zc = np.array([oz + ozs * dz], dtype=np.float32)
            xc = np.array([ox + oxs * dx], dtype=np.float32)
            for lst, grid in zip(lists, _four_grids(zc, xc, hypers, nts, method, nfilt, dipole, zds, xds)):
                lst.append(grid)
            oxs = oxs + spacing
    return lists[0], lists[1], lists[2], lists[3], sourceAxis


def buildReceiversGeometry(parObject, elasticParam):
    """Receivers on the four staggered grids (constant geometry for all shots).
    Returns (center, x, z, xz) lists and the receiver axis."""
    if isinstance(parObject, dict):
        parObject = paramObj(parObject)
    dipole = parObject.getInt("dipole", 0)
    zds = parObject.getFloat("zDipoleShift", 0.0)
    xds = parObject.getFloat("xDipoleShift", 0.0)
    nts = parObject.getInt("nts")
    h = elasticParam.getHyper()
    dz, oz = h.getAxis(1).d, h.getAxis(1).o
    dx, ox = h.getAxis(2).d, h.getAxis(2).o
    hypers = _staggered_hypers(elasticParam)
    method = parObject.getString("recInterpMethod", "linear")
    nfilt = parObject.getInt("recInterpNumFilters", 4)
    geom = parObject.getString("recGeomFile", "none")
    if geom != "none":
        g = _geometry_array(geom)
        xc = np.ascontiguousarray(g[0, :, 0], dtype=np.float32)
        zc = np.ascontiguousarray(g[2, :, 0], dtype=np.float32)
        nRec = parObject.getInt("nReceiver")
        if nRec != len(xc):
            raise ValueError("ERROR [buildReceiversGeometry]: Number of receiver coordinates (%s) not consistent "
                             "with parameter file (nReceiver=%d)" % (len(xc), nRec))
        receiverAxis = axis(nRec, 1.0, 1.0)
    else:
        ozr = parObject.getInt("depthReceiver") - 1 + parObject.getInt("zPadMinus") + parObject.getInt("fat", 4)
        nxr = parObject.getInt("nReceiver")
        oxr = parObject.getInt("oReceiver") - 1 + parObject.getInt("xPadMinus") + parObject.getInt("fat", 4)
        dxr = parObject.getInt("dReceiver")
        receiverAxis = axis(nxr, ox + oxr * dx, dxr * dx)
        irec = np.arange(nxr, dtype=np.float64)
        zc = np.empty(nxr, dtype=np.float32)
        xc = np.empty(nxr, dtype=np.float32)
        # float32 element-wise assignment like the SepVector ndarray writes
        zc[:] = oz + ozr * dz + 0 * dz * irec
        xc[:] = ox + oxr * dx + dxr * dx * irec
    grids = _four_grids(zc, xc, hypers, nts, method, nfilt, dipole, zds, xds)
    return [grids[0]], [grids[1]], [grids[2]], [grids[3]], receiverAxis
