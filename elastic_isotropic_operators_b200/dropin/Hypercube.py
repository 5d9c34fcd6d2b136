"""``Hypercube`` of SEP's Python stack: axes (n, o, d, label, unit) and
hypercubes (axis 1 fastest, getAxis 1-based), as the reference's scripts
build them (Hypercube.axis(n=, o=, d=), Hypercube.hypercube(axes=[...]))."""
from _eio_dropin import sepvec


class axis(sepvec.axis):
    pass


class hypercube(sepvec.hypercube):
    def getCpp(self):
        return self


__all__ = ["axis", "hypercube"]
