"""Shared helpers of the parity tests: regular-grid inputs prepared by the
oracle, and calls of the product's single-shot C entry points."""
import ctypes

import numpy as np

from elastic_isotropic_operators_b200 import _lib, prop
from oracle import oracle as O

FIELD_GRID = O.FIELD_GRID


def reg_inputs(w, prec="f", shot=0, seed=11, method="linear", nfilt=1):
    """Regular-grid inputs of one shot of workload ``w``: grid dict, medium,
    position lists, random source/data traces and the fine-time Born source."""
    orc = O.Oracle(prec)
    c = O.Case.from_workload(w, method, nfilt)
    g = c.grid()
    med = orc.medium(c.ep, g["dts"], g["S"])
    src = O._grids(orc, c, *c.src[shot])
    rec = O._grids(orc, c, *c.rec)
    sp = [G["uniq"].astype(np.int32) for G in src]
    rp = [G["uniq"].astype(np.int32) for G in rec]
    rng = np.random.default_rng(seed)
    nts = g["nts"]
    model = [rng.standard_normal((len(sp[FIELD_GRID[f]]), nts)).astype(orc.dt) for f in range(5)]
    data = [rng.standard_normal((len(rp[FIELD_GRID[f]]), nts)).astype(orc.dt) for f in range(5)]
    fine = O.born_sources(orc, c, g, med, src, w.source_signal().reshape(5, 1, nts))
    dm = [rng.standard_normal((w.nx, w.nz)).astype(orc.dt) * 1e-3 for _ in range(5)]
    return dict(orc=orc, case=c, g=g, med=med, sp=sp, rp=rp, model=model, data=data, fine=fine, dm=dm)


class Ctx:
    """Product context (eio_ctx) of workload ``w`` on cuda:0."""

    def __init__(self, w):
        self.L = _lib.lib()
        self.fd = prop.fd_params_from_par(w.par, w.elastic)
        ep = np.ascontiguousarray(w.elastic.getNdArray(), np.float32)
        h = ctypes.c_void_p()
        _lib.check(self.L.eio_ctx_create(ctypes.byref(self.fd), _lib.fptr(ep), 0, ctypes.byref(h)))
        self.h = h

    def set_kernel(self, kind, tz=64, cw=8, cpr=8):
        _lib.check(self.L.eio_ctx_set_kernel(self.h, kind, tz, cw, cpr))

    def get_kernel(self):
        v = [ctypes.c_int() for _ in range(4)]
        _lib.check(self.L.eio_ctx_get_kernel(self.h, *[ctypes.byref(x) for x in v]))
        return tuple(x.value for x in v)

    def autotune(self):
        v = [ctypes.c_int() for _ in range(4)]
        _lib.check(self.L.eio_ctx_autotune(self.h, *[ctypes.byref(x) for x in v]))
        return tuple(x.value for x in v)

    def close(self):
        if self.h is not None:
            self.L.eio_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    @staticmethod
    def _pos(pl):
        arrs = [np.ascontiguousarray(p, np.int32) for p in pl]
        return arrs, _lib.ptr_array([a.ctypes.data for a in arrs]), (ctypes.c_int * 4)(*[len(a) for a in arrs])

    def nl(self, adj, model, data, sp, rp):
        model = [np.ascontiguousarray(m, np.float32) for m in model]
        data = [np.ascontiguousarray(d, np.float32) for d in data]
        sa, spp, sn = self._pos(sp)
        ra, rpp, rn = self._pos(rp)
        fn = self.L.eio_nl_adj_reg if adj else self.L.eio_nl_fwd_reg
        _lib.check(fn(self.h, _lib.ptr_array([m.ctypes.data for m in model]),
                      _lib.ptr_array([d.ctypes.data for d in data]), spp, sn, rpp, rn))
        return model, data

    def born(self, adj, fine, dm, data, sp, rp):
        fine = [np.ascontiguousarray(f, np.float32) for f in fine]
        dm = [np.ascontiguousarray(d, np.float32) for d in dm]
        data = [np.ascontiguousarray(d, np.float32) for d in data]
        sa, spp, sn = self._pos(sp)
        ra, rpp, rn = self._pos(rp)
        fn = self.L.eio_born_adj_reg if adj else self.L.eio_born_fwd_reg
        _lib.check(fn(self.h, _lib.ptr_array([f.ctypes.data for f in fine]), _lib.ptr_array([d.ctypes.data for d in dm]),
                      _lib.ptr_array([d.ctypes.data for d in data]), spp, sn, rpp, rn))
        return dm, data


def rel(a, b):
    return O.rel_l2(np.concatenate([np.ravel(x) for x in a]), np.concatenate([np.ravel(x) for x in b]))
