"""SEP ``.H`` file input/output without genericIO.

The reference reads and writes its models, wavelets and data through SEP's
genericIO (``genericIO.defaultIO.getVector`` / ``writeVector``).  A SEP
dataset is a text header plus a raw binary file:

* the header is a history of ``key=value`` pairs (several per line, values
  optionally quoted, later occurrences override earlier ones); ``n1..nk``,
  ``o1..ok``, ``d1..dk``, ``label1..``, ``unit1..`` describe the axes (axis 1
  fastest), ``in=`` names the binary file and ``data_format`` its encoding;
* the binary holds the samples with axis 1 fastest: ``xdr_float`` is
  big-endian float32, ``native_float`` little-endian float32, ``xdr_double``
  / ``native_double`` the 64-bit versions.

``readSep`` returns a ``sepvec.floatVector`` (numpy shape = reversed axes), so
files written by the reference's tools load directly into the operators here;
``writeSep`` writes the same layout.
"""
import os
import re

import numpy as np

from .sepvec import axis, doubleVector, floatVector, hypercube

__all__ = ["parse_header", "readSep", "writeSep"]

_FORMATS = {
    "xdr_float": np.dtype(">f4"),
    "native_float": np.dtype("<f4"),
    "xdr_double": np.dtype(">f8"),
    "native_double": np.dtype("<f8"),
}

_PAIR = re.compile(r"""([A-Za-z_][A-Za-z0-9_.]*)=("[^"]*"|'[^']*'|\S*)""")


def parse_header(text):
    """Dictionary of the ``key=value`` pairs of a SEP header (last one wins)."""
    out = {}
    for line in text.splitlines():
        for key, val in _PAIR.findall(line):
            if len(val) >= 2 and val[0] == val[-1] and val[0] in "\"'":
                val = val[1:-1]
            out[key] = val
    return out


def _axes(h, ndims=None):
    k = 1
    while "n%d" % (k + 1) in h:
        k += 1
    while k > 1 and int(h.get("n%d" % k, 1)) == 1:
        k -= 1
    if ndims is not None:
        k = max(k, int(ndims))
    axes = []
    for i in range(1, k + 1):
        axes.append(axis(int(h.get("n%d" % i, 1)), float(h.get("o%d" % i, 0.0)), float(h.get("d%d" % i, 1.0)),
                         h.get("label%d" % i, ""), h.get("unit%d" % i, "")))
    return axes


def _binary_path(header_path, h):
    if "in" not in h:
        raise IOError("SEP header %s has no in= entry" % header_path)
    path = h["in"]
    if os.path.isabs(path) and os.path.exists(path):
        return path
    cand = os.path.join(os.path.dirname(os.path.abspath(header_path)), os.path.basename(path))
    if os.path.exists(cand):
        return cand
    if os.path.exists(path):
        return path
    raise IOError("binary %s of SEP header %s not found" % (path, header_path))


def readSep(path, ndims=None):
    """Read a SEP dataset; ``ndims`` keeps trailing axes of length one."""
    with open(path) as f:
        h = parse_header(f.read())
    fmt = h.get("data_format", "xdr_float")
    if fmt not in _FORMATS:
        raise IOError("unsupported SEP data_format %s" % fmt)
    axes = _axes(h, ndims)
    count = int(np.prod([a.n for a in axes]))
    raw = np.fromfile(_binary_path(path, h), dtype=_FORMATS[fmt], count=count)
    if raw.size != count:
        raise IOError("SEP binary of %s holds %d samples, the header describes %d" % (path, raw.size, count))
    cls = floatVector if _FORMATS[fmt].itemsize == 4 else doubleVector
    return cls(hypercube(axes=axes), raw.astype(cls.dtype))


def writeSep(path, vec, data_format="xdr_float", binary=None):
    """Write ``vec`` (a sepvec vector) as ``path`` + binary (default ``path@``)."""
    if data_format not in _FORMATS:
        raise ValueError("unsupported SEP data_format %s" % data_format)
    binary = binary or path + "@"
    hyper = vec.getHyper()
    arr = np.ascontiguousarray(vec.getNdArray(), dtype=_FORMATS[data_format])
    arr.tofile(binary)
    lines = ["", "elastic_isotropic_operators_b200.sepio.writeSep"]
    for i, a in enumerate(hyper.axes, start=1):
        lines.append('\tn%d=%d  o%d=%.9g  d%d=%.9g  label%d="%s"  unit%d="%s"' %
                     (i, a.n, i, a.o, i, a.d, i, a.label, i, a.unit))
    lines.append("\tesize=%d" % _FORMATS[data_format].itemsize)
    lines.append('\tdata_format="%s"' % data_format)
    lines.append("in=%s" % binary)
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")
    return path
