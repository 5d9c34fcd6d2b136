"""``genericIO`` of SEP's Python stack, as the reference's scripts use it:

* ``io(params=sys.argv)``: the parameters of a run -- ``key=value`` arguments,
  with every ``par=file`` argument replaced by the ``key=value`` pairs of that
  parameter file at its place (later values override earlier ones) -- with
  getInt / getFloat / getString / getInts / getFloats / getBool;
* ``defaultIO.getVector(file, ndims=None)`` / ``defaultIO.writeVector(file,
  vec)``: SEP ``.H`` datasets (header + binary; xdr or native floats).
"""
import os

from _eio_dropin import sepio, sepvec


def _pairs(tokens, depth=0):
    out = {}
    for tok in tokens:
        if "=" not in tok:
            continue                       # the program name, flags
        k, v = tok.split("=", 1)
        k, v = k.strip(), v.strip().strip('"').strip("'")
        if k == "par":
            if depth > 8:
                raise ValueError("par files nest too deeply")
            with open(v) as f:
                toks = []
                for line in f.read().splitlines():
                    toks.extend(line.split("#", 1)[0].split())
            out.update(_pairs(toks, depth + 1))
        else:
            out[k] = v
    return out


class io(sepvec.paramObj):
    """Parameters of a run (see the module docstring); also reads and writes
    SEP datasets like ``defaultIO``."""

    def __init__(self, params=None, **kw):
        if isinstance(params, dict):
            super().__init__(params)
        else:
            super().__init__(_pairs(list(params or [])))
        self._d.update({k: str(v) for k, v in kw.items()})

    def getFloats(self, key, default=None):
        def conv(v):
            if isinstance(v, (list, tuple)):
                return [float(x) for x in v]
            return [float(x) for x in str(v).split(",") if x.strip()]
        return self._get(key, default, conv)

    def getBool(self, key, default=None):
        return self._get(key, default, lambda v: str(v).strip().lower() in ("1", "y", "yes", "true", "t"))

    def getCpp(self):
        return self

    @staticmethod
    def getVector(filename, ndims=None):
        return sepio.readSep(os.fspath(filename), ndims)

    @staticmethod
    def writeVector(filename, vec):
        sepio.writeSep(os.fspath(filename), vec)


class _DefaultIO:
    getVector = staticmethod(io.getVector)
    writeVector = staticmethod(io.writeVector)


defaultIO = _DefaultIO()

__all__ = ["io", "defaultIO"]
