"""Minimal stand-ins for the SEP vector stack the reference operators take.

The reference's pybind11 classes accept ``SEP::float3DReg`` / ``float4DReg``
vectors, ``SEP::hypercube`` and ``paramObj`` (genericIO / sepVector, not
vendored with the reference).  These classes provide the part of that API the
operator path uses: axes with (n, o, d), numpy-backed storage whose numpy
shape is the axis list reversed (axis 1 fastest), ``getNdArray``,
``getHyper``, ``clone``, ``scale``, ``dot``, ``rand``/``random``, ``writeVec``, and a
``paramObj`` with ``getInt``/``getFloat``/``getString``/``getInts`` over a
par-file or a dict.
"""
import numpy as np


class axis:
    def __init__(self, n=1, o=0.0, d=1.0, label="", unit=""):
        self.n = int(n)
        self.o = float(o)
        self.d = float(d)
        self.label = label
        self.unit = unit

    def __repr__(self):
        return "axis(n=%d, o=%g, d=%g)" % (self.n, self.o, self.d)


class hypercube:
    def __init__(self, axes=None, ns=None, os=None, ds=None):
        if axes is None:
            ns = list(ns)
            os = list(os) if os is not None else [0.0] * len(ns)
            ds = list(ds) if ds is not None else [1.0] * len(ns)
            axes = [axis(n, o, d) for n, o, d in zip(ns, os, ds)]
        self.axes = [axis(a.n, a.o, a.d, a.label, a.unit) for a in axes]

    def getAxis(self, i):
        """1-based, like SEP::hypercube::getAxis."""
        return self.axes[i - 1]

    def getNs(self):
        return [a.n for a in self.axes]

    def getNdim(self):
        return len(self.axes)

    def getN123(self):
        return int(np.prod(self.getNs()))

    def clone(self):
        return hypercube(axes=self.axes)

    def checkSame(self, other):
        return all(a.n == b.n and abs(a.o - b.o) < 1e-6 and abs(a.d - b.d) < 1e-6
                   for a, b in zip(self.axes, other.axes)) and len(self.axes) == len(other.axes)


class floatVector:
    """numpy-backed vector; numpy shape = reversed axis sizes (axis 1 fastest)."""

    dtype = np.float32

    def __init__(self, hyper, arr=None):
        self.hyper = hyper
        shape = tuple(reversed(hyper.getNs()))
        if arr is None:
            self.arr = np.zeros(shape, dtype=self.dtype)
        else:
            arr = np.ascontiguousarray(arr, dtype=self.dtype)
            if arr.size != int(np.prod(shape)):
                raise ValueError("array size does not match the hypercube")
            self.arr = arr.reshape(shape)

    def getNdArray(self):
        return self.arr

    def getHyper(self):
        return self.hyper

    def getCpp(self):
        return self

    def clone(self):
        return type(self)(self.hyper.clone(), self.arr.copy())

    def cloneSpace(self):
        return type(self)(self.hyper.clone())

    def zero(self):
        self.arr[...] = 0
        return self

    def set(self, v):
        self.arr[...] = v
        return self

    def scale(self, s):
        self.arr *= self.dtype(s) if self.dtype == np.float64 else s
        return self

    def rand(self, seed=None):
        rng = np.random.default_rng(seed)
        self.arr[...] = rng.uniform(-1.0, 1.0, size=self.arr.shape).astype(self.dtype)
        return self

    random = rand

    def dot(self, other):
        return float(np.dot(self.arr.ravel().astype(np.float64), other.arr.ravel().astype(np.float64)))

    def norm(self):
        return float(np.sqrt(self.dot(self)))

    def checkSame(self, other):
        return self.hyper.checkSame(other.hyper)

    def writeVec(self, filename, data_format="xdr_float"):
        """Write the vector as a SEP dataset (``filename`` header + ``filename@`` binary)."""
        from .sepio import writeSep
        writeSep(filename, self, data_format)


class doubleVector(floatVector):
    dtype = np.float64


def getSepVector(hyper=None, ns=None, storage="dataFloat", axes=None):
    if hyper is None:
        hyper = hypercube(axes=axes) if axes is not None else hypercube(ns=ns)
    if storage == "dataDouble":
        return doubleVector(hyper)
    return floatVector(hyper)


class paramObj:
    """Par-file parameters (``key=value`` lines, ``#`` comments) or a dict."""

    def __init__(self, params=None, text=None):
        self.param = self
        self._d = {}
        if text is not None:
            for line in text.splitlines():
                line = line.split("#", 1)[0]
                for tok in line.split():
                    if "=" in tok:
                        k, v = tok.split("=", 1)
                        self._d[k.strip()] = v.strip().strip('"')
        if params:
            for k, v in params.items():
                self._d[k] = v

    @classmethod
    def from_file(cls, path):
        with open(path) as f:
            return cls(text=f.read())

    def _get(self, key, default, conv):
        if key in self._d:
            return conv(self._d[key])
        if default is None:
            raise KeyError("missing parameter: %s" % key)
        return default

    def getInt(self, key, default=None):
        return self._get(key, default, lambda v: int(float(v)))

    def getFloat(self, key, default=None):
        return self._get(key, default, float)

    def getString(self, key, default=None):
        return self._get(key, default, str)

    def getInts(self, key, default=None):
        def conv(v):
            if isinstance(v, (list, tuple)):
                return [int(x) for x in v]
            return [int(x) for x in str(v).split(",") if x.strip()]
        return self._get(key, default, conv)

    def has(self, key):
        return key in self._d

    def set(self, key, value):
        self._d[key] = value

    def as_dict(self):
        return dict(self._d)
