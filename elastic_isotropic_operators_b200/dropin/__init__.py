"""Drop-in modules for the reference's Python scripts.

The reference's scripts (nonlinearPythonElasticFloatMain.py,
BornPythonElasticFloatMain.py, efwiMain.py, ...) import the pybind11 modules
``pyElastic_iso_float_nl`` / ``pyElastic_iso_float_born``, the wrapper module
``Elastic_iso_float_prop`` and SEP's Python stack (``genericIO``,
``SepVector``, ``Hypercube``, ``pyOperator``, ``elasticParamConvertModule``,
``pyDaskOperator``).  This directory holds modules under exactly those names,
built on this package's operators, so those scripts run unchanged once the
directory is first on the module search path::

    PYTHONPATH=<repo>/elastic_isotropic_operators_b200/dropin python3 nonlinearPythonElasticFloatMain.py par=...

or, from Python, ``elastic_isotropic_operators_b200.dropin.activate()``.

Only the part of the SEP stack those scripts use is provided (SEP ``.H``
files through ``sepio``, par files and command-line parameters, vectors and
hypercubes from ``sepvec``, the pySolver operator base class with its dot
test).  Dask clusters are not: one process per GPU with torch.distributed
(``shots.ShotParallel``) replaces them, and a script that asks for a Dask
client gets an error naming that.
"""
import os
import sys

DIR = os.path.dirname(os.path.abspath(__file__))

__all__ = ["DIR", "activate"]


def activate():
    """Put the drop-in modules first on ``sys.path`` (idempotent)."""
    if sys.path[:1] != [DIR]:
        while DIR in sys.path:
            sys.path.remove(DIR)
        sys.path.insert(0, DIR)
    return DIR
