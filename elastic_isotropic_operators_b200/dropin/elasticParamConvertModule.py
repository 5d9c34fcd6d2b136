"""``elasticParamConvertModule`` (seis_utils/python/elasticParamConvertModule.py:5-117):
the parameter conversion and its Jacobian as pySolver operators over the
elastic-model vector, on fwi.ElasticConv / fwi.ElasticConvJab."""
from _eio_dropin import fwi
from pyOperator import Operator


class ElasticConv(Operator):
    """conv_type 1: VpVsRho (m/s, m/s, kg/m3) -> RhoLameMu (kg/m3, Pa, Pa);
    2: from km/s, km/s, g/cm3; -1: RhoLameMu -> VpVsRho."""

    def __init__(self, domain, conv_type):
        super().__init__(domain, domain)
        self._op = fwi.ElasticConv(conv_type)

    def forward(self, add, model, data):
        self._op.forward(add, model, data)


class ElasticConvJab(Operator):
    """Jacobian of the VpVsRho -> RhoLameMu conversion at ``background``."""

    def __init__(self, domain, background, conv_type):
        super().__init__(domain, domain)
        self._op = fwi.ElasticConvJab(background, conv_type)

    def forward(self, add, model, data):
        self._op.forward(add, model, data)

    def adjoint(self, add, model, data):
        self._op.adjoint(add, model, data)

    def setBackground(self, background):
        self._op.setBackground(background)


__all__ = ["ElasticConv", "ElasticConvJab"]
