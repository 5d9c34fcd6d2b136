"""Born operators with shots in lockstep (eio_ctx_set_born_batch > 1): the
shots of a call run in groups, one k_step_shots launch per fine
step for every shot of a group (the shots of a tile next to each other, one
copy of the medium), the imaging of a group's shots in one launch.

Each shot's arithmetic is that of the one-shot tile kernel, so with the same
kernel kind (k_step at 4 CTAs per SM) the forward traces of every shot are
bitwise equal to the shots run one at a time on the lanes; the adjoint image
sums the shots in another order (each shot of a group images into its own
buffer) and agrees to 1e-6.  Both agree with the oracle to 1e-5.  Covered:
uneven groups (5 shots in groups of 3 and 2), add, cropped shots of different
windows, the device-pointer entry eio_born_shots_dev."""
import ctypes

import numpy as np
import pytest

from elastic_isotropic_operators_b200 import _lib, prop, synthetic
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL32 = 1e-5


def _ops(w, batch):
    src, rec = w.geometry()
    born = prop.BornElasticShotsGpu(w.elastic, w.par, [w.source_signal()], *src, *rec)
    born.setBornBatch(batch)
    born.setLanes(3)
    _lib.check(born._L.eio_ctx_set_kernel(born.ctx, 3, 64, 16, 0))
    return born


def _lanes(op):
    lanes, active = ctypes.c_int(), ctypes.c_int()
    _lib.check(op._L.eio_ctx_get_lanes(op.ctx, ctypes.byref(lanes), ctypes.byref(active)))
    return active.value


def test_batched_born_equals_one_shot_at_a_time_and_oracle():
    w = synthetic.small(nts=120, nshots=5)
    one, bat = _ops(w, 1), _ops(w, 3)
    dm = one.modelSpace()
    dm.getNdArray()[...] = w.extra["dmodel"]
    d1, d3 = one.dataSpace(), bat.dataSpace()
    one.forward(False, dm, d1)
    bat.forward(False, dm, d3)
    assert _lanes(bat) == 3
    assert np.array_equal(d1.getNdArray(), d3.getNdArray())          # per-shot arithmetic unchanged
    c = O.Case.from_workload(w)
    want = O.born_forward(O.Oracle("f"), c, dm.getNdArray(), [w.source_signal()])
    assert O.rel_l2(d3.getNdArray(), want) < TOL32
    # add accumulates
    d3b = bat.dataSpace()
    d3b.getNdArray()[...] = 1.0
    bat.forward(True, dm, d3b)
    assert np.allclose(d3b.getNdArray(), d3.getNdArray() + 1.0, rtol=0, atol=1e-6)
    # adjoint
    rng = np.random.default_rng(3)
    data = one.dataSpace()
    data.getNdArray()[...] = rng.standard_normal(data.getNdArray().shape).astype(np.float32)
    g1, g3 = one.modelSpace(), bat.modelSpace()
    one.adjoint(False, g1, data)
    bat.adjoint(False, g3, data)
    assert O.rel_l2(g3.getNdArray(), g1.getNdArray()) < 1e-6
    gwant = O.born_adjoint(O.Oracle("f"), c, data.getNdArray(), [w.source_signal()])
    assert O.rel_l2(g3.getNdArray(), gwant) < TOL32
    assert bat.dotTest(False, 1e-5), bat.lastDotTest


def test_batched_born_with_cropped_shots():
    """Shots of one group on different windows (different tile counts)."""
    import test_windows as TW
    w, src_x, recs = TW._case()
    outs = []
    for batch in (1, 2):
        src, rec = TW._geometry(w, w.elastic, src_x, recs, [0, 1])
        born = prop.BornElasticShotsGpu(w.elastic, w.par, [w.source_signal()], *src, *rec)
        born.setBornBatch(batch)
        born.setShotWindows([24, 104], [88, 120])
        _lib.check(born._L.eio_ctx_set_kernel(born.ctx, 3, 64, 16, 0))
        dm = born.modelSpace()
        dm.getNdArray()[...] = w.extra["dmodel"]
        d = born.dataSpace()
        born.forward(False, dm, d)
        rng = np.random.default_rng(5)
        dd = born.dataSpace()
        dd.getNdArray()[...] = rng.standard_normal(dd.getNdArray().shape).astype(np.float32)
        g = born.modelSpace()
        born.adjoint(False, g, dd)
        outs.append((d.getNdArray().copy(), g.getNdArray().copy()))
    assert np.array_equal(outs[0][0], outs[1][0])
    assert O.rel_l2(outs[1][1], outs[0][1]) < 1e-6


def test_batched_born_device_entry_matches_oracle():
    """eio_born_shots_dev (device-resident traces, no receiver interpolation)."""
    torch = pytest.importorskip("torch")
    from helpers import reg_inputs
    w = synthetic.small(nts=100, nshots=3)
    born = _ops(w, 3)
    L, ctx = born._L, born.ctx
    shots = [reg_inputs(w, "f", shot=e, seed=9) for e in range(w.nExp)]
    dev = torch.device("cuda")
    dm5 = [torch.from_numpy(np.ascontiguousarray(a)).to(dev) for a in shots[0]["dm"]]
    grad5 = [torch.zeros_like(a) for a in dm5]
    fine = [[torch.from_numpy(np.ascontiguousarray(f)).to(dev) for f in r["fine"]] for r in shots]
    data = [[torch.zeros((len(r["rp"][O.FIELD_GRID[f]]), w.nts), dtype=torch.float32, device=dev)
             for f in range(5)] for r in shots]
    keep = []

    def pa(lst):
        arrs = [np.ascontiguousarray(p, np.int32) for p in lst]
        keep.append(arrs)
        return arrs

    sp = [pa(r["sp"]) for r in shots]
    rp = [pa(r["rp"]) for r in shots]
    args = (_lib.ptr_array([t.data_ptr() for s in fine for t in s]),
            _lib.ptr_array([t.data_ptr() for t in dm5]),
            _lib.ptr_array([t.data_ptr() for s in data for t in s]),
            _lib.ptr_array([a.ctypes.data for s in sp for a in s]),
            (ctypes.c_int * (4 * len(sp)))(*[len(a) for s in sp for a in s]),
            _lib.ptr_array([a.ctypes.data for s in rp for a in s]),
            (ctypes.c_int * (4 * len(rp)))(*[len(a) for s in rp for a in s]))
    _lib.check(L.eio_born_shots_dev(ctx, 0, w.nExp, *args))
    torch.cuda.synchronize()
    orc = shots[0]["orc"]
    for e, r in enumerate(shots):
        dm_ref = [x.copy() for x in r["dm"]]
        d_ref = [np.zeros_like(x) for x in r["data"]]
        orc.born_prop(0, r["g"], r["med"], r["fine"], dm_ref, d_ref, r["sp"], r["rp"])
        got = [t.cpu().numpy() for t in data[e]]
        assert O.rel_l2(np.concatenate([x.ravel() for x in got]),
                        np.concatenate([x.ravel() for x in d_ref])) < TOL32, e
    # adjoint of those traces into grad5 (summed over the shots)
    args_adj = (args[0], _lib.ptr_array([t.data_ptr() for t in grad5])) + args[2:]
    _lib.check(L.eio_born_shots_dev(ctx, 1, w.nExp, *args_adj))
    torch.cuda.synchronize()
    want = [np.zeros_like(x) for x in shots[0]["dm"]]
    for e, r in enumerate(shots):
        d_in = [t.cpu().numpy() for t in data[e]]
        orc.born_prop(1, r["g"], r["med"], r["fine"], want, d_in, r["sp"], r["rp"])
    got = np.concatenate([t.cpu().numpy().ravel() for t in grad5])
    assert O.rel_l2(got, np.concatenate([x.ravel() for x in want])) < TOL32


@pytest.mark.parametrize("nshots,batch", [(3, 3), (5, 2)])
def test_persistent_time_loop_equals_per_step_launches(nshots, batch):
    """The shot groups' persistent loop (one launch per propagation phase, tiles
    advancing behind per-tile step counters, secondary sources computed per
    tile) gives the bits of the per-step launches, forward and adjoint."""
    w = synthetic.small(nts=90, nshots=nshots)
    out = []
    for persistent in (0, 7):
        op = _ops(w, batch)
        op.setPersistent(persistent)
        dm = op.modelSpace()
        dm.getNdArray()[...] = w.extra["dmodel"]
        d = op.dataSpace()
        op.forward(False, dm, d)
        rng = np.random.default_rng(7)
        dd = op.dataSpace()
        dd.getNdArray()[...] = rng.standard_normal(dd.getNdArray().shape).astype(np.float32)
        g = op.modelSpace()
        op.adjoint(False, g, dd)
        out.append((d.getNdArray().copy(), g.getNdArray().copy()))
    assert np.abs(out[0][0]).max() > 0
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])
