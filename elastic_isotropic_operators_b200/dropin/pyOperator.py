"""``pyOperator`` of the pySolver stack, the part the reference's wrappers
and scripts use: the ``Operator`` base class (domain and range spaces, the
dot-product test) and ``ChainOperator`` (B after A)."""
import numpy as np


def _nd(v):
    return v.getNdArray() if hasattr(v, "getNdArray") else np.asarray(v)


def _dot64(a, b):
    return float(np.dot(_nd(a).ravel().astype(np.float64), _nd(b).ravel().astype(np.float64)))


class Operator:
    def __init__(self, domain=None, range=None):
        if domain is not None and range is not None:
            self.setDomainRange(domain, range)

    def setDomainRange(self, domain, range):
        """Keep zeroed vectors shaped like ``domain`` and ``range``."""
        self.domain = domain.cloneSpace() if hasattr(domain, "cloneSpace") else domain
        self.range = range.cloneSpace() if hasattr(range, "cloneSpace") else range

    def getDomain(self):
        return self.domain

    def getRange(self):
        return self.range

    def forward(self, add, model, data):
        raise NotImplementedError("forward of %s" % type(self).__name__)

    def adjoint(self, add, model, data):
        raise NotImplementedError("adjoint of %s" % type(self).__name__)

    def dotTest(self, verb=False, maxError=1e-4):
        """<A x, y> against <x, A^T y> for random x, y (FP64 sums), with add
        off and on; raises RuntimeError when a relative error exceeds maxError.
        The add pass starts from the outputs of the first pass, so the
        accumulated vectors keep the operator's own scale (an O(1) random start
        would swamp a small-valued output in FP32)."""
        x = self.domain.clone().rand()
        y = self.range.clone().rand()
        Ax = self.range.clone().zero()
        ATy = self.domain.clone().zero()
        results = []
        for add in (False, True):
            ax0, aty0 = Ax.clone(), ATy.clone()
            self.forward(add, x, Ax)
            self.adjoint(add, ATy, y)
            lhs = _dot64(Ax, y) - (_dot64(ax0, y) if add else 0.0)
            rhs = _dot64(x, ATy) - (_dot64(x, aty0) if add else 0.0)
            err = abs(lhs - rhs) / max(abs(lhs), abs(rhs), 1e-300)
            results.append(err)
            if verb:
                print("Dot-product test (add=%s): <Ax,y> = %.10e, <x,A'y> = %.10e, relative error %.3e"
                      % (add, lhs, rhs, err))
        if max(results) > maxError:
            raise RuntimeError("dot-product test failed: relative errors %s above %g" % (results, maxError))
        return results


class ChainOperator(Operator):
    """C = B A: forward A then B, adjoint B^T then A^T."""

    def __init__(self, A, B):
        super().__init__(A.getDomain(), B.getRange())
        self.A, self.B = A, B
        self._tmp = A.getRange().clone()

    def forward(self, add, model, data):
        self.A.forward(False, model, self._tmp)
        self.B.forward(add, self._tmp, data)

    def adjoint(self, add, model, data):
        self.B.adjoint(False, self._tmp, data)
        self.A.adjoint(add, model, self._tmp)


__all__ = ["Operator", "ChainOperator"]
