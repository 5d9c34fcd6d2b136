"""Imports this package from the drop-in modules, which are loaded by their
bare names (the drop-in directory on sys.path, the package's parent maybe not)."""
import os
import sys

try:
    import elastic_isotropic_operators_b200 as eio  # noqa: F401
except ImportError:   # the drop-in directory alone is on the path
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))))
    import elastic_isotropic_operators_b200 as eio  # noqa: F401

from elastic_isotropic_operators_b200 import fwi, prop, sepio, sepvec  # noqa: E402,F401
