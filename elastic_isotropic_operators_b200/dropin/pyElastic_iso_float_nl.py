"""``pyElastic_iso_float_nl`` (python_float/pyElastic_iso_float_nl.cpp:15-57):
``spaceInterpGpu``, ``nonlinearPropElasticShotsGpu`` and ``ostream_redirect``
with the pybind11 module's constructor arguments and methods, on this
package's sm_100a engine (elastic_isotropic_operators_b200.prop).

    spaceInterpGpu(zCoord, xCoord, gridHyper, nt, method, nFilt, dipole, zDipoleShift, xDipoleShift)
    nonlinearPropElasticShotsGpu(elasticParam, par, srcCenter, srcX, srcZ, srcXZ, recCenter, recX, recZ, recXZ)
        .forward(add, model, data) / .adjoint / .forwardWavefield / .adjointWavefield
        .getWavefield() / .setBackground(elasticParam) / .dotTest(verbose, maxError)

Errors come back as exceptions (EioError, a RuntimeError) where the
reference's C++ throws std::runtime_error or exits the process."""
import contextlib

from _eio_dropin import prop

spaceInterpGpu = prop.spaceInterpGpu
nonlinearPropElasticShotsGpu = prop.nonlinearPropElasticShotsGpu


@contextlib.contextmanager
def ostream_redirect(stdout=True, stderr=True):
    """The engine writes nothing to the C++ streams: nothing to redirect."""
    yield


__all__ = ["spaceInterpGpu", "nonlinearPropElasticShotsGpu", "ostream_redirect"]
