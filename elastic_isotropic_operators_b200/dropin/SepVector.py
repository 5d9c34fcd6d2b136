"""``SepVector`` of SEP's Python stack: numpy-backed float/double vectors over
a hypercube (numpy shape = axes reversed, axis 1 fastest) with getNdArray,
getHyper, getCpp, clone, zero, scale, dot, norm, rand and writeVec (a SEP
``.H`` file through sepio)."""
from _eio_dropin import sepvec


def _hyper(hyper=None, ns=None, axes=None):
    if hyper is not None:
        return hyper
    if axes is not None:
        return sepvec.hypercube(axes=axes)
    return sepvec.hypercube(ns=ns)


class floatVector(sepvec.floatVector):
    """floatVector(hyper=...), floatVector(fromCpp=vector) (shares the storage,
    like the pybind wrapper of a C++ vector) or floatVector(hyper, array)."""

    def __init__(self, hyper=None, arr=None, fromCpp=None, **kw):
        if fromCpp is not None:
            super().__init__(fromCpp.getHyper(), None)
            self.arr = fromCpp.getNdArray()
            return
        super().__init__(_hyper(hyper, kw.get("ns"), kw.get("axes")), arr)


class doubleVector(floatVector):
    dtype = sepvec.doubleVector.dtype


def getSepVector(hyper=None, ns=None, storage="dataFloat", axes=None):
    """A zeroed vector over ``hyper`` (or axes / ns); storage dataFloat or dataDouble."""
    h = _hyper(hyper, ns, axes)
    return doubleVector(h) if storage == "dataDouble" else floatVector(h)


__all__ = ["floatVector", "doubleVector", "getSepVector"]
