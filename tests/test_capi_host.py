"""CPU tests of the C ABI: the library loads, exports every entry point that
include/eio_b200.h declares, and its host-side preparation (medium, staggering,
spatial and temporal interpolation, QC) agrees bit for bit with the oracle.
No propagation is run here (that needs the GPU)."""
import ctypes
import os
import re

import numpy as np
import pytest

from elastic_isotropic_operators_b200 import _lib, prop, synthetic
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    text = open(os.path.join(ROOT, "include", "eio_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(eio_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    names = header_symbols()
    assert len(names) >= 30
    for n in names:
        assert hasattr(L, n), n
    assert set(names) == set(_lib.exported_symbols())
    assert L.eio_version() >= 1


def test_medium_matches_oracle_bitwise(small_case):
    w = small_case
    fd = prop.fd_params_from_par(w.par, w.elastic)
    ep = np.ascontiguousarray(w.elastic.getNdArray(), np.float32)
    out = [np.zeros((w.nx, w.nz), np.float32) for _ in range(5)]
    _lib.check(_lib.lib().eio_medium_prepare(ctypes.byref(fd), _lib.fptr(ep), *[_lib.fptr(o) for o in out]))
    ref = O.Oracle("f").medium(ep, w.dts, 2 * w.sub)
    for a, b in zip(out, ref):
        np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("axis_", [0, 1])
@pytest.mark.parametrize("adj", [0, 1])
def test_stagger_matches_oracle(axis_, adj):
    rng = np.random.default_rng(5)
    m = rng.standard_normal((19, 23)).astype(np.float32)
    d = rng.standard_normal((19, 23)).astype(np.float32)
    m1, d1, m2, d2 = m.copy(), d.copy(), m.copy(), d.copy()
    _lib.check(_lib.lib().eio_stagger(axis_, adj, 1, 23, 19, _lib.fptr(m1), _lib.fptr(d1)))
    O.Oracle("f").stagger(axis_, adj, 1, m2, d2)
    np.testing.assert_array_equal(m1, m2)
    np.testing.assert_array_equal(d1, d2)


@pytest.mark.parametrize("adj", [0, 1])
def test_time_interp_matches_oracle(adj):
    rng = np.random.default_rng(6)
    nts, S = 37, 4
    ntw = (nts - 1) * S + 1
    c = rng.standard_normal((3, nts)).astype(np.float32)
    f = rng.standard_normal((3, ntw)).astype(np.float32)
    c1, f1, c2, f2 = c.copy(), f.copy(), c.copy(), f.copy()
    _lib.check(_lib.lib().eio_time_interp(adj, 1, nts, 1e-3, 0.0, S, 3, _lib.fptr(c1), _lib.fptr(f1)))
    O.Oracle("f").tinterp(adj, 1, nts, 1e-3, 0.0, S, c2, f2)
    np.testing.assert_array_equal(c1, c2)
    np.testing.assert_array_equal(f1, f2)


@pytest.mark.parametrize("method,nfilt", [("linear", 1), ("sinc", 1), ("sinc", 2), ("gauss", 1)])
def test_space_interp_matches_oracle(method, nfilt):
    rng = np.random.default_rng(7)
    zc = rng.uniform(60, 400, 11).astype(np.float32)
    xc = rng.uniform(60, 600, 11).astype(np.float32)
    hyp = prop.hypercube(axes=[prop.axis(60, -5.0, 10.0), prop.axis(80, -5.0, 10.0)])
    s = prop.spaceInterpGpu(zc, xc, hyp, 13, method, nfilt, 0, 0.0, 0.0)
    o = O.Oracle("f").sinterp(zc, xc, 60, -5.0, 10.0, 80, -5.0, 10.0, method, nfilt)
    np.testing.assert_array_equal(s.getRegPosUnique(), o["uniq"])
    gpi, w = s.getWeights()
    np.testing.assert_array_equal(gpi, o["gpi"])
    np.testing.assert_allclose(w, o["w"], rtol=2e-7, atol=0)
    reg = rng.standard_normal((s.nDeviceReg, 13)).astype(np.float32)
    irr = np.zeros((11, 13), np.float32)
    s.forward(False, reg, irr)
    irr2 = np.zeros((11, 13), np.float32)
    O.Oracle("f").sinterp_apply(o, 0, 0, reg.copy(), irr2)
    np.testing.assert_allclose(irr, irr2, rtol=1e-6, atol=1e-6)


def test_space_interp_dipole_and_errors():
    hyp = prop.hypercube(axes=[prop.axis(60, 0.0, 10.0), prop.axis(80, 0.0, 10.0)])
    s = prop.spaceInterpGpu(np.float32([200.0]), np.float32([300.0]), hyp, 5, "linear", 1, 1, 1.0, 0.0)
    assert s.nFiltTotal == 8
    _, w = s.getWeights()
    assert abs(w.sum()) < 1e-6     # a dipole integrates to zero
    with pytest.raises(prop.EioError):
        prop.spaceInterpGpu(np.float32([2.0]), np.float32([300.0]), hyp, 5, "linear", 1, 0, 0.0, 0.0)
    with pytest.raises(prop.EioError):
        prop.spaceInterpGpu(np.float32([200.0]), np.float32([300.0]), hyp, 5, "sinc", 1, 1, 0.0, 0.0)
    with pytest.raises(prop.EioError):
        prop.spaceInterpGpu(np.float32([200.0]), np.float32([300.0]), hyp, 5, "cubic", 1, 0, 0.0, 0.0)


def test_qc_errors_come_back_as_status(small_case):
    w = small_case
    L = _lib.lib()
    ep = np.ascontiguousarray(w.elastic.getNdArray(), np.float32)
    out = [np.zeros((w.nx, w.nz), np.float32) for _ in range(5)]
    fd = prop.fd_params_from_par(w.par, w.elastic)
    fd.dts = 0.01   # Courant far above 0.45
    st = L.eio_medium_prepare(ctypes.byref(fd), _lib.fptr(ep), *[_lib.fptr(o) for o in out])
    assert st == -2 and b"Courant" in L.eio_last_error()
    fd = prop.fd_params_from_par(w.par, w.elastic)
    fd.fMax = 500.0
    st = L.eio_medium_prepare(ctypes.byref(fd), _lib.fptr(ep), *[_lib.fptr(o) for o in out])
    assert st == -2 and b"Dispersion" in L.eio_last_error()
    fd = prop.fd_params_from_par(w.par, w.elastic)
    fd.nz = w.nz - 4
    st = L.eio_medium_prepare(ctypes.byref(fd), _lib.fptr(ep[:, :, :w.nz - 4].copy()), *[_lib.fptr(o) for o in out])
    assert st == -2
    fd = prop.fd_params_from_par(w.par, w.elastic)
    fd.sub = 60
    st = L.eio_medium_prepare(ctypes.byref(fd), _lib.fptr(ep), *[_lib.fptr(o) for o in out])
    assert st == -2 and b"SUB_MAX" in L.eio_last_error()


@pytest.mark.parametrize("param,ix,iz,value", [(0, 0, 0, np.nan), (1, 50, 30, np.inf), (2, 103, 71, -np.inf)])
def test_non_finite_medium_is_rejected_with_its_cell(small_case, param, ix, iz, value):
    """A NaN or Inf anywhere in the elastic parameters (pads included: every
    cell enters the stencil) is an argument error naming the parameter and the
    cell, before the QC (whose comparisons a NaN would slip through)."""
    w = small_case
    L = _lib.lib()
    ep = np.ascontiguousarray(w.elastic.getNdArray(), np.float32).copy()
    ep[param, ix, iz] = value
    out = [np.zeros((w.nx, w.nz), np.float32) for _ in range(5)]
    fd = prop.fd_params_from_par(w.par, w.elastic)
    st = L.eio_medium_prepare(ctypes.byref(fd), _lib.fptr(ep), *[_lib.fptr(o) for o in out])
    msg = L.eio_last_error().decode()
    assert st == -1, msg
    assert ("rho", "lambda", "mu")[param] in msg and "ix=%d, iz=%d" % (ix, iz) in msg


def test_device_memory_cap_is_process_wide_and_host_only_to_set():
    L = _lib.lib()
    used = ctypes.c_longlong(-1)
    _lib.check(L.eio_get_device_memory_used(ctypes.byref(used)))
    assert used.value >= 0
    _lib.check(L.eio_set_device_memory_cap(1 << 20))
    _lib.check(L.eio_set_device_memory_cap(0))


def test_no_cpu_fallback_without_gpu(small_case):
    """Without a usable CUDA device the engine fails loudly (no CPU path)."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    w = small_case
    src, rec = w.geometry()
    with pytest.raises(prop.EioError) as e:
        prop.nonlinearPropElasticShotsGpu(w.elastic, w.par, *src, *rec)
    assert e.value.code == -3
