"""``pyElastic_iso_float_born`` (python_float/pyElastic_iso_float_born.cpp:15-40):
``BornElasticShotsGpu(elasticParam, par, sourcesSignals, srcCenter, srcX,
srcZ, srcXZ, recCenter, recX, recZ, recXZ)`` with forward(add, model, data),
adjoint(add, model, data) and setBackground(elasticParam), on this package's
sm_100a engine (elastic_isotropic_operators_b200.prop)."""
from _eio_dropin import prop
from pyElastic_iso_float_nl import ostream_redirect  # noqa: F401  (the module exports it too)

BornElasticShotsGpu = prop.BornElasticShotsGpu

__all__ = ["BornElasticShotsGpu", "ostream_redirect"]
