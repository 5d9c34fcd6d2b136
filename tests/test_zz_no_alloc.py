"""Allocation-free nonlinear forward propagation (eio_nl_fwd_noalloc).

Some callers cannot call cudaMalloc: their device memory belongs to another
allocator, they forbid allocation once they are running, or they must not
grow the device footprint of the process that loads them.  For them the
library keeps all scratch of one nonlinear forward propagation in a fixed
device array of its own, and the caller passes only inputs and outputs.

The test runs that entry point through the C ABI twice in a row with
different source traces and compares each result with the allocating entry
point eio_nl_fwd_reg_dev, so scratch left over from the first call would
show up in the second.  It lives in a file of its own that pytest collects
last, and it runs the same alone in a fresh process or after the other tests.
"""
import ctypes

import numpy as np
import pytest

from elastic_isotropic_operators_b200 import _lib, prop, synthetic

from helpers import Ctx, reg_inputs, rel

pytestmark = pytest.mark.gpu

TOL = 1e-5   # the FP32 parity tolerance of the other GPU tests


def _pp(tensors):
    return _lib.ptr_array([t.data_ptr() for t in tensors])


def _positions(pl):
    arrs = [np.ascontiguousarray(p, np.int32) for p in pl]
    return arrs, _lib.ptr_array([a.ctypes.data for a in arrs]), (ctypes.c_int * 4)(*[len(a) for a in arrs])


def test_noalloc_matches_allocating_entry_point():
    import torch
    w = synthetic.small()
    r = reg_inputs(w, "f", seed=41)
    L = _lib.lib()
    dev = torch.device("cuda", 0)
    fd = prop.fd_params_from_par(w.par, w.elastic)
    ep = np.ascontiguousarray(w.elastic.getNdArray(), np.float32)
    med = [np.zeros((w.nx, w.nz), np.float32) for _ in range(5)]
    _lib.check(L.eio_medium_prepare(ctypes.byref(fd), _lib.fptr(ep), *[_lib.fptr(m) for m in med]))
    med_d = [torch.from_numpy(m).to(dev) for m in med]
    sa, spp, sn = _positions(r["sp"])
    ra, rpp, rn = _positions(r["rp"])
    ctx = Ctx(w)   # the allocating path, same tile kernel
    try:
        ctx.set_kernel(0)
        rng = np.random.default_rng(3)
        for call in range(2):
            model = [rng.standard_normal(m.shape).astype(np.float32) for m in r["model"]]
            model_d = [torch.from_numpy(m).to(dev) for m in model]
            want_d = [torch.zeros(d.shape, dtype=torch.float32, device=dev) for d in r["data"]]
            got_d = [torch.full(d.shape, 7.0, dtype=torch.float32, device=dev) for d in r["data"]]
            _lib.check(L.eio_nl_fwd_reg_dev(ctx.h, _pp(model_d), _pp(want_d), spp, sn, rpp, rn))
            _lib.check(L.eio_nl_fwd_noalloc(ctypes.byref(fd), _pp(med_d), _pp(model_d), _pp(got_d), spp, sn, rpp,
                                            rn, None))
            torch.cuda.synchronize()
            want = [t.cpu().numpy() for t in want_d]
            got = [t.cpu().numpy() for t in got_d]
            assert max(float(np.abs(x).max()) for x in want) > 0
            assert rel(got, want) < TOL, (call, rel(got, want))
    finally:
        ctx.close()


def test_noalloc_rejects_sizes_beyond_its_limit():
    import torch
    w = synthetic.small()
    L = _lib.lib()
    fd = prop.fd_params_from_par(w.par, w.elastic)
    fd.nz, fd.nx = 520, 1016          # 528,320 cells > 262,144
    dummy = [torch.zeros(16, device="cuda") for _ in range(5)]
    zero_pos = (ctypes.c_int * 4)(0, 0, 0, 0)
    nulls = _lib.ptr_array([0, 0, 0, 0])
    st = L.eio_nl_fwd_noalloc(ctypes.byref(fd), _pp(dummy), _pp(dummy), _pp(dummy), nulls, zero_pos, nulls,
                              zero_pos, None)
    assert st == -1
    assert b"allocation-free limit" in L.eio_last_error()
