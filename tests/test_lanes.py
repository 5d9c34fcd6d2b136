"""Shot lanes: the multi-shot operators spread their shots over several engines
of one GPU.  Per-shot outputs do not depend on the lane count (bitwise: each
shot runs the same kernels on its own engine); stacked outputs (the Born image,
the constant-source nonlinear adjoint) are sums in another order (relative L2
<= 1e-6).  The device-resident multi-shot entry point equals shot-by-shot calls."""
import ctypes

import numpy as np
import pytest
import torch

from elastic_isotropic_operators_b200 import _lib, prop, synthetic

from helpers import reg_inputs

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a, b = np.ravel(a).astype(np.float64), np.ravel(b).astype(np.float64)
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def _run(w, lanes):
    src, rec = w.geometry()
    nl = prop.nonlinearPropElasticShotsGpu(w.elastic, w.par, *src, *rec)
    born = prop.BornElasticShotsGpu(w.elastic, w.par, [w.source_signal()], *src, *rec)
    out = {}
    for op in (nl, born):
        _lib.check(op._L.eio_ctx_set_kernel(op.ctx, 3, 64, 16, 0))
        _lib.check(op._L.eio_ctx_set_lanes(op.ctx, lanes))
    rng = np.random.default_rng(5)
    m = nl.modelSpace()
    m.getNdArray()[...] = w.source_signal()[None]
    d = nl.dataSpace()
    nl.forward(False, m, d)
    out["nl_fwd"] = d.getNdArray().copy()
    r = nl.dataSpace()
    r.getNdArray()[...] = rng.standard_normal(r.getNdArray().shape).astype(np.float32)
    ma = nl.modelSpace()
    nl.adjoint(False, ma, r)
    out["nl_adj"] = ma.getNdArray().copy()
    dm = born.modelSpace()
    dm.getNdArray()[...] = w.extra["dmodel"]
    bd = born.dataSpace()
    born.forward(False, dm, bd)
    out["born_fwd"] = bd.getNdArray().copy()
    g = born.modelSpace()
    born.adjoint(False, g, r)
    out["born_adj"] = g.getNdArray().copy()
    act = ctypes.c_int()
    _lib.check(born._L.eio_ctx_get_lanes(born.ctx, None, ctypes.byref(act)))
    out["active"] = act.value
    return out


def test_lane_count_does_not_change_results():
    w = synthetic.small(nts=60, nshots=5)
    one = _run(w, 1)
    assert one["active"] == 1
    for lanes in (2, 3):
        many = _run(w, lanes)
        assert many["active"] == lanes
        assert np.array_equal(many["nl_fwd"], one["nl_fwd"])
        assert np.array_equal(many["born_fwd"], one["born_fwd"])
        assert _rel(many["nl_adj"], one["nl_adj"]) < 1e-6
        assert _rel(many["born_adj"], one["born_adj"]) < 1e-6


def test_born_shots_dev_equals_shot_by_shot():
    w = synthetic.small(nts=60, nshots=3)
    src, rec = w.geometry()
    born = prop.BornElasticShotsGpu(w.elastic, w.par, [w.source_signal()], *src, *rec)
    L, ctx = born._L, born.ctx
    _lib.check(L.eio_ctx_set_kernel(ctx, 3, 64, 16, 0))
    dev = torch.device("cuda", 0)
    dm5 = [torch.from_numpy(a).to(dev) for a in born.prepareModel(w.extra["dmodel"])]
    shots = []
    for e in range(w.nExp):
        fine, sp, rp = born.prepareShot(e)
        shots.append(dict(fine=[torch.from_numpy(a).to(dev) for a in fine],
                          sp=[np.ascontiguousarray(p, np.int32) for p in sp],
                          rp=[np.ascontiguousarray(p, np.int32) for p in rp]))
    nrec = [len(p) for p in shots[0]["rp"]]

    def data():
        return [[torch.zeros((nrec[prop._FIELD_GRID[f]], w.nts), device=dev) for f in range(5)] for _ in shots]

    pp = lambda ts: _lib.ptr_array([t.data_ptr() for t in ts])
    # shot by shot on one lane
    d1 = data()
    g1 = [torch.zeros_like(a) for a in dm5]
    for s, d in zip(shots, d1):
        args = (pp(s["fine"]), None, pp(d), _lib.ptr_array([a.ctypes.data for a in s["sp"]]),
                (ctypes.c_int * 4)(*[len(a) for a in s["sp"]]), _lib.ptr_array([a.ctypes.data for a in s["rp"]]),
                (ctypes.c_int * 4)(*[len(a) for a in s["rp"]]))
        _lib.check(L.eio_born_fwd_reg_dev(ctx, args[0], pp(dm5), *args[2:]))
    for s, d in zip(shots, d1):
        _lib.check(L.eio_born_adj_reg_dev(ctx, pp(s["fine"]), pp(g1), pp(d),
                                          _lib.ptr_array([a.ctypes.data for a in s["sp"]]),
                                          (ctypes.c_int * 4)(*[len(a) for a in s["sp"]]),
                                          _lib.ptr_array([a.ctypes.data for a in s["rp"]]),
                                          (ctypes.c_int * 4)(*[len(a) for a in s["rp"]])))
    # all shots in one call on two lanes
    _lib.check(L.eio_ctx_set_lanes(ctx, 2))
    d2 = data()
    g2 = [torch.zeros_like(a) for a in dm5]
    all_fine = _lib.ptr_array([t.data_ptr() for s in shots for t in s["fine"]])
    all_data = _lib.ptr_array([t.data_ptr() for d in d2 for t in d])
    all_sp = _lib.ptr_array([a.ctypes.data for s in shots for a in s["sp"]])
    all_sn = (ctypes.c_int * (4 * len(shots)))(*[len(a) for s in shots for a in s["sp"]])
    all_rp = _lib.ptr_array([a.ctypes.data for s in shots for a in s["rp"]])
    all_rn = (ctypes.c_int * (4 * len(shots)))(*[len(a) for s in shots for a in s["rp"]])
    _lib.check(L.eio_born_shots_dev(ctx, 0, len(shots), all_fine, pp(dm5), all_data, all_sp, all_sn, all_rp, all_rn))
    _lib.check(L.eio_born_shots_dev(ctx, 1, len(shots), all_fine, pp(g2), all_data, all_sp, all_sn, all_rp, all_rn))
    torch.cuda.synchronize()
    for a, b in zip(d1, d2):
        for x, y in zip(a, b):
            assert torch.equal(x, y)
    for x, y in zip(g1, g2):
        assert _rel(y.cpu().numpy(), x.cpu().numpy()) < 1e-6
