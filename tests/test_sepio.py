"""SEP .H input/output (the genericIO getVector / writeVector the reference's
scripts use to load models, wavelets and data)."""
import numpy as np
import pytest

from elastic_isotropic_operators_b200 import sepio
from elastic_isotropic_operators_b200.sepvec import axis, floatVector, hypercube


@pytest.mark.parametrize("fmt", ["xdr_float", "native_float"])
def test_round_trip(tmp_path, fmt):
    rng = np.random.default_rng(1)
    hyp = hypercube(axes=[axis(7, 0.0, 10.0, "z", "m"), axis(5, -20.0, 10.0, "x", "m"), axis(3)])
    v = floatVector(hyp, rng.standard_normal((3, 5, 7)).astype(np.float32))
    p = sepio.writeSep(str(tmp_path / "m.H"), v, data_format=fmt)
    w = sepio.readSep(p)
    assert np.array_equal(w.getNdArray(), v.getNdArray())
    assert [(a.n, a.o, a.d) for a in w.getHyper().axes] == [(7, 0.0, 10.0), (5, -20.0, 10.0), (3, 0.0, 1.0)]
    assert w.getHyper().getAxis(1).label == "z"
    raw = np.fromfile(str(tmp_path / "m.H@"), dtype=">f4" if fmt == "xdr_float" else "<f4")
    assert np.array_equal(raw, v.getNdArray().ravel())


def test_history_header_last_value_wins(tmp_path):
    """A header with an older history block: the later n/o/d, in= and
    data_format entries override the earlier ones; trailing n=1 axes drop."""
    data = (np.arange(4 * 6 * 3, dtype=np.float32) * 0.5 + 1500.0).reshape(3, 6, 4)
    data.astype(">f4").tofile(str(tmp_path / "layers.H@"))
    text = "\n".join([
        "", "Build:   user@host   Mon Jan  1 00:00:00 2024",
        '\t\tsets next: in="/elsewhere/tmp@abc"',
        "\tn1=9  o1=0.0  d1=1.0",
        "\tn2=6  o2=0.000000  d2=10.000000   label2=\"Undefined\"   unit2=\"Undefined\"",
        "\tn3=3  o3=0.000000  d3=10.000000",
        "hff=-1 gff=-1  n4=1  n5=1  n6=1  n7=1  n8=1  n9=1 ",
        "\tn1=4  o1=0.000000  d1=10.000000   label1=\"Undefined\"   unit1=\"Undefined\"",
        "\t\tesize=4", '\t\tdata_format="xdr_float"', "", "",
        "Smooth:   user@host   Mon Jan  1 00:00:01 2024",
        '\t\tsets next: in="/elsewhere/smooth@def"', "\t\tData smoothed with: rect1=10",
        '\t\tdata_format="xdr_float"', "in=./layers.H@", ""])
    (tmp_path / "layers.H").write_text(text)
    h = sepio.parse_header(text)
    assert h["n1"] == "4" and h["in"] == "./layers.H@" and h["rect1"] == "10"
    v = sepio.readSep(str(tmp_path / "layers.H"))
    assert v.getHyper().getNs() == [4, 6, 3]
    assert np.array_equal(v.getNdArray(), data)
    assert sepio.readSep(str(tmp_path / "layers.H"), ndims=5).getHyper().getNs() == [4, 6, 3, 1, 1]


def test_errors(tmp_path):
    (tmp_path / "a.H").write_text("n1=10 data_format=\"xdr_float\" in=./a.H@\n")
    np.zeros(4, ">f4").tofile(str(tmp_path / "a.H@"))
    with pytest.raises(IOError):
        sepio.readSep(str(tmp_path / "a.H"))             # short binary
    (tmp_path / "b.H").write_text("n1=4 data_format=\"xdr_int\" in=./a.H@\n")
    with pytest.raises(IOError):
        sepio.readSep(str(tmp_path / "b.H"))
    (tmp_path / "c.H").write_text("n1=4\n")
    with pytest.raises(IOError):
        sepio.readSep(str(tmp_path / "c.H"))


def test_model_file_feeds_medium_preparation(tmp_path):
    """A (rho, lambda, mu) model written as SEP goes through the library's
    medium preparation unchanged."""
    import ctypes
    from elastic_isotropic_operators_b200 import _lib, prop, synthetic
    w = synthetic.small()
    p = sepio.writeSep(str(tmp_path / "ela.H"), w.elastic)
    ep = sepio.readSep(p)
    assert np.array_equal(ep.getNdArray(), w.elastic.getNdArray())
    fd = prop.fd_params_from_par(w.par, ep)
    out = [np.zeros((w.nx, w.nz), np.float32) for _ in range(5)]
    arr = np.ascontiguousarray(ep.getNdArray(), np.float32)
    _lib.check(_lib.lib().eio_medium_prepare(ctypes.byref(fd), _lib.fptr(arr), *[_lib.fptr(o) for o in out]))
    assert all(np.isfinite(o).all() for o in out)


@pytest.mark.parametrize("surface", [0, 1])
def test_padding_rule(surface):
    """padElasticFileGpuMain: block-multiple interiors, edge replication,
    fat-only top pad with the free surface."""
    from elastic_isotropic_operators_b200 import padding
    rng = np.random.default_rng(2)
    nz, nx = 37, 53
    hyp = hypercube(axes=[axis(nz, 100.0, 5.0), axis(nx, -50.0, 5.0), axis(3)])
    v = floatVector(hyp, rng.uniform(1, 2, (3, nx, nz)).astype(np.float32))
    out, pads = padding.padElasticFile(v, 20, 30, surfaceCondition=surface)
    a = out.getNdArray()
    nzN, nxN = a.shape[2], a.shape[1]
    assert (nzN - 8) % 16 == 0 and (nxN - 8) % 16 == 0
    zm = pads["zPadMinus"]
    assert zm == (4 if surface else 20) and pads["xPadMinus"] == 30
    assert nzN == zm + pads["zPadPlus"] + nz + 8 and nxN == 30 + pads["xPadPlus"] + nx + 8
    z0, x0 = 4 + zm, 34
    m = v.getNdArray()
    assert np.array_equal(a[:, x0:x0 + nx, z0:z0 + nz], m)
    assert np.array_equal(a[:, x0:x0 + nx, 0], m[:, :, 0]) and np.array_equal(a[:, x0:x0 + nx, -1], m[:, :, -1])
    assert np.array_equal(a[:, 0], a[:, x0]) and np.array_equal(a[:, -1], a[:, x0 + nx - 1])
    assert abs(out.getHyper().getAxis(1).o - (100.0 - z0 * 5.0)) < 1e-9
    assert abs(out.getHyper().getAxis(2).o - (-50.0 - x0 * 5.0)) < 1e-9
    if surface:
        assert z0 == 8      # the free surface row 2*fat holds the first model row
