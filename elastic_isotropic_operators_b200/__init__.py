"""B200-native (sm_100a) 2-D isotropic elastic staggered-grid FD engine.

Drop-in for the propagation path of biondiettore/elastic_isotropic_operators:
nonlinear shot modelling, the Born operator over (drho, dlambda, dmu) and both
adjoints, behind the reference's operator API (``prop``) and a C ABI
(``include/eio_b200.h``, ``libeio_b200.so``).
"""
from ._lib import EioError, LIB_PATH  # noqa: F401

__all__ = ["EioError", "LIB_PATH", "prop", "sepvec", "synthetic"]
