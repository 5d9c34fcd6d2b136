"""``Elastic_iso_float_prop`` (python_float/Elastic_iso_float_prop.py): the
operator set-up functions and pySolver operator wrappers of the reference's
Python layer, on this package's sm_100a engine.

* ``nonlinearOpInitFloat(args)`` (:842-932), ``nonlinearFwiOpInitFloat(args)``
  (:1012-1104), ``BornOpInitFloat(args)`` (:1155-1252): read the parameters
  (``par=`` files and ``key=value`` arguments), the elastic model
  (``elasticParam=``, converted from VpVsRho when ``mod_par`` != 0), the source
  signals where the operator needs them (``sources=``), build the
  staggered-grid source and receiver geometry and allocate the model and data
  vectors; they return the same tuples as the reference's functions.
* ``nonlinearPropElasticShotsGpu``, ``nonlinearFwiPropElasticShotsGpu``,
  ``BornElasticShotsGpu`` (:935-1311): ``pyOperator.Operator`` subclasses
  with the reference's constructor arguments (domain, range, then the pybind
  class's arguments), unwrapping ``getCpp()`` vectors like the reference.
* ``buildSourceGeometry`` / ``buildReceiversGeometry`` (:205-364, 525-661),
  ``parfile2pars``, ``create_parObj``, ``call_spaceInterpGpu``,
  ``create_client``.

Dask clusters (``hostnames=``, ``pbs_args=``, ``lsf_args=``) are not
supported: ``create_client`` raises and names the replacement (one process
per GPU under torch.distributed, ``shots.ShotParallel``).  Without them
``create_client`` returns (None, None) and every set-up function takes the
reference's single-process path.
"""
import re

import numpy as np

import genericIO
import Hypercube
import SepVector
import elasticParamConvertModule as ElaConv
import pyElastic_iso_float_born
import pyElastic_iso_float_nl
import pyOperator as Op
from _eio_dropin import prop
from pyElastic_iso_float_nl import spaceInterpGpu

__all__ = ["create_client", "parfile2pars", "create_parObj", "call_spaceInterpGpu", "buildSourceGeometry",
           "buildReceiversGeometry", "nonlinearOpInitFloat", "nonlinearPropElasticShotsGpu",
           "nonlinearFwiOpInitFloat", "nonlinearFwiPropElasticShotsGpu", "BornOpInitFloat", "BornElasticShotsGpu"]


def _cpp(v):
    return v.getCpp() if hasattr(v, "getCpp") else v


# ----------------------------------------------------------------------- helpers
def create_client(parObject):
    """(None, None): this engine runs without Dask; a requested cluster raises."""
    for key in ("hostnames", "pbs_args", "lsf_args"):
        if parObject.getString(key, "none") not in ("none", "noHost", "noPBS", "noLSF"):
            raise NotImplementedError(
                "%s= asks for a Dask cluster, which this engine does not use: run one process per GPU with "
                "torch.distributed (elastic_isotropic_operators_b200.shots.ShotParallel)" % key)
    return None, None


def parfile2pars(args):
    """``args`` with its last ``par=file`` argument replaced by that file's lines."""
    args = list(args)
    found = [i for i, a in enumerate(args) if re.match(r"^par=", a)]
    if not found:
        return args
    i = found[-1]
    with open(args[i].split("=", 1)[1]) as f:
        lines = f.read().splitlines()
    return args[:i] + lines + args[i + 1:]


def create_parObj(args):
    return genericIO.io(params=args)


def call_spaceInterpGpu(zAxes, xAxes, zCoord, xCoord, GridAxes, nts, sourceInterpMethod, sourceInterpNumFilters,
                        dipole, zDipoleShift, xDipoleShift):
    """A spaceInterpGpu over the grid of ``GridAxes`` for the coordinates zCoord, xCoord."""
    grid = Hypercube.hypercube(axes=GridAxes)
    z = SepVector.getSepVector(axes=zAxes)
    x = SepVector.getSepVector(axes=xAxes)
    z.getNdArray()[:] = zCoord
    x.getNdArray()[:] = xCoord
    return spaceInterpGpu(z.getCpp(), x.getCpp(), grid.getCpp(), nts, sourceInterpMethod, sourceInterpNumFilters,
                          dipole, zDipoleShift, xDipoleShift)


def buildSourceGeometry(parObject, elasticParam):
    """(center, x-shifted, z-shifted, xz-shifted source lists, shot axis)."""
    return prop.buildSourceGeometry(parObject, elasticParam)


def buildReceiversGeometry(parObject, elasticParam):
    """(center, x-shifted, z-shifted, xz-shifted receiver lists, receiver axis)."""
    return prop.buildReceiversGeometry(parObject, elasticParam)


def _time_axis(par):
    return Hypercube.axis(n=par.getInt("nts", -1), o=par.getFloat("ots", 0.0), d=par.getFloat("dts", -1.0))


def _elastic_file(par):
    name = par.getString("elasticParam", "noElasticParamFile")
    if name == "noElasticParamFile":
        raise IOError("**** ERROR: User did not provide elastic parameter file ****")
    return genericIO.defaultIO.getVector(name)


def _to_rho_lame_mu(par, elastic, in_place):
    """mod_par 1 / 2: VpVsRho (m/s or km/s units) -> rho, lambda, mu; 0: as given."""
    mod_par = par.getInt("mod_par", 0)
    if mod_par == 0:
        return elastic
    conv = ElaConv.ElasticConv(elastic, mod_par)
    if in_place:
        src = elastic.clone()
        conv.forward(False, src, elastic)
        return elastic
    out = elastic.clone()
    conv.forward(False, elastic, out)
    return out


def _no_client(client):
    if client:
        raise NotImplementedError("Dask clients are not supported (see create_client)")


def _sources_file(par, ndims=3):
    name = par.getString("sources", "noSourcesFile")
    if name == "noSourcesFile":
        raise IOError("**** ERROR: User did not provide seismic sources file ****")
    return genericIO.defaultIO.getVector(name, ndims=ndims)


def _data_vector(par, elastic, time_axis):
    src = buildSourceGeometry(par, elastic)
    rec = buildReceiversGeometry(par, elastic)
    hyper = Hypercube.hypercube(axes=[time_axis, rec[4], Hypercube.axis(n=5), src[4]])
    return src[:4], rec[:4], SepVector.getSepVector(hyper, storage="dataFloat")


# ----------------------------------------------------------------------- nonlinear
def nonlinearOpInitFloat(args, client=None):
    """Set-up of the nonlinear operator (Elastic_iso_float_prop.py:842-932).
    Returns modelFloat, dataFloat, elasticParamFloat, parObject, the 8
    geometry lists (sources center/x/z/xz, receivers center/x/z/xz) and
    modelFloatLocal (the same vector as modelFloat without Dask)."""
    _no_client(client)
    par = genericIO.io(params=args)
    t = _time_axis(par)
    dummy, comps = Hypercube.axis(n=1), Hypercube.axis(n=5)
    geom = par.getString("sourceGeomFile", "None")
    if geom != "None":
        sim = genericIO.defaultIO.getVector(geom, ndims=3).getHyper().getAxis(2)
        model_axes = [t, Hypercube.axis(n=sim.n, o=sim.o, d=sim.d), comps, dummy]
    else:
        model_axes = [t, dummy, comps, dummy]
    model = SepVector.getSepVector(Hypercube.hypercube(axes=model_axes), storage="dataFloat")
    elastic = _to_rho_lame_mu(par, _elastic_file(par), in_place=True)
    src, rec, data = _data_vector(par, elastic, t)
    return (model, data, elastic, par) + tuple(src) + tuple(rec) + (model,)


class nonlinearPropElasticShotsGpu(Op.Operator):
    """Nonlinear operator (source signals -> data) as a pySolver operator."""

    def __init__(self, domain, range, elasticParam, paramP, sourcesVectorCenterGrid, sourcesVectorXGrid,
                 sourcesVectorZGrid, sourcesVectorXZGrid, receiversVectorCenterGrid, receiversVectorXGrid,
                 receiversVectorZGrid, receiversVectorXZGrid):
        self.setDomainRange(domain, range)
        self.pyOp = pyElastic_iso_float_nl.nonlinearPropElasticShotsGpu(
            _cpp(elasticParam), _cpp(paramP).param, sourcesVectorCenterGrid, sourcesVectorXGrid, sourcesVectorZGrid,
            sourcesVectorXZGrid, receiversVectorCenterGrid, receiversVectorXGrid, receiversVectorZGrid,
            receiversVectorXZGrid)

    def __str__(self):
        return " NLOper "

    def forward(self, add, model, data):
        with pyElastic_iso_float_nl.ostream_redirect():
            self.pyOp.forward(add, _cpp(model), _cpp(data))

    def forwardWavefield(self, add, model, data):
        with pyElastic_iso_float_nl.ostream_redirect():
            self.pyOp.forwardWavefield(add, _cpp(model), _cpp(data))

    def adjoint(self, add, model, data):
        with pyElastic_iso_float_nl.ostream_redirect():
            self.pyOp.adjoint(add, _cpp(model), _cpp(data))

    def adjointWavefield(self, add, model, data):
        with pyElastic_iso_float_nl.ostream_redirect():
            self.pyOp.adjointWavefield(add, _cpp(model), _cpp(data))

    def getWavefield(self):
        return SepVector.floatVector(fromCpp=self.pyOp.getWavefield())

    def setBackground(self, elasticParam):
        with pyElastic_iso_float_nl.ostream_redirect():
            self.pyOp.setBackground(_cpp(elasticParam))

    def dotTestCpp(self, verb=False, maxError=.00001):
        """The engine's own dot-product test (FP64 reductions on the GPU)."""
        with pyElastic_iso_float_nl.ostream_redirect():
            return self.pyOp.dotTest(verb, maxError)


def nonlinearFwiOpInitFloat(args, client=None):
    """Set-up of the nonlinear FWI operator (elastic model -> data, fixed
    sources; Elastic_iso_float_prop.py:1012-1104).  Returns elasticParamFloat
    (as read), elasticParamFloatConv (rho, lambda, mu), dataFloat, sourceFloat,
    parObject, the 8 geometry lists and elasticParamFloatLocal."""
    _no_client(client)
    par = genericIO.io(params=args)
    elastic = _elastic_file(par)
    elastic_conv = _to_rho_lame_mu(par, elastic, in_place=False)
    t = _time_axis(par)
    dummy, comps = Hypercube.axis(n=1), Hypercube.axis(n=5)
    source = SepVector.getSepVector(Hypercube.hypercube(axes=[t, dummy, comps, dummy]), storage="dataFloat")
    source.getNdArray()[0, :, 0, :] = np.asarray(_sources_file(par).getNdArray()).reshape(5, -1)
    src, rec, data = _data_vector(par, elastic, t)
    return (elastic, elastic_conv, data, source, par) + tuple(src) + tuple(rec) + (elastic,)


class nonlinearFwiPropElasticShotsGpu(Op.Operator):
    """Nonlinear FWI operator: forward(add, model, data) sets ``model`` (rho,
    lambda, mu) as the background and propagates the fixed ``sources``."""

    def __init__(self, domain, range, sources, paramP, sourcesVectorCenterGrid, sourcesVectorXGrid,
                 sourcesVectorZGrid, sourcesVectorXZGrid, receiversVectorCenterGrid, receiversVectorXGrid,
                 receiversVectorZGrid, receiversVectorXZGrid):
        self.setDomainRange(domain, range)
        self.sources = _cpp(sources).clone()
        self.pyOp = pyElastic_iso_float_nl.nonlinearPropElasticShotsGpu(
            _cpp(domain), _cpp(paramP).param, sourcesVectorCenterGrid, sourcesVectorXGrid, sourcesVectorZGrid,
            sourcesVectorXZGrid, receiversVectorCenterGrid, receiversVectorXGrid, receiversVectorZGrid,
            receiversVectorXZGrid)

    def __str__(self):
        return " NLOper "

    def forward(self, add, model, data):
        self.setBackground(model)
        with pyElastic_iso_float_nl.ostream_redirect():
            self.pyOp.forward(add, self.sources, _cpp(data))

    def setBackground(self, elasticParam):
        with pyElastic_iso_float_nl.ostream_redirect():
            self.pyOp.setBackground(_cpp(elasticParam))


# ----------------------------------------------------------------------- Born
def BornOpInitFloat(args, client=None):
    """Set-up of the Born operator (Elastic_iso_float_prop.py:1155-1252).
    Returns modelFloat (zeroed, the elastic model's space), dataFloat,
    elasticParamFloat (rho, lambda, mu), parObject, sourcesSignalsVector (one
    signal for every shot), the 8 geometry lists and modelFloatLocal."""
    _no_client(client)
    par = genericIO.io(params=args)
    elastic = _to_rho_lame_mu(par, _elastic_file(par), in_place=True)
    t = _time_axis(par)
    signals = [_sources_file(par)]
    model = SepVector.getSepVector(elastic.getHyper(), storage="dataFloat")
    src, rec, data = _data_vector(par, elastic, t)
    return (model, data, elastic, par, signals) + tuple(src) + tuple(rec) + (model,)


class BornElasticShotsGpu(Op.Operator):
    """Born operator (drho, dlambda, dmu -> data) as a pySolver operator."""

    def __init__(self, domain, range, elasticParam, paramP, sourcesSignalsVector, sourcesVectorCenterGrid,
                 sourcesVectorXGrid, sourcesVectorZGrid, sourcesVectorXZGrid, receiversVectorCenterGrid,
                 receiversVectorXGrid, receiversVectorZGrid, receiversVectorXZGrid):
        self.setDomainRange(domain, range)
        signals = [_cpp(s) for s in sourcesSignalsVector]
        self.pyOp = pyElastic_iso_float_born.BornElasticShotsGpu(
            _cpp(elasticParam), _cpp(paramP).param, signals, sourcesVectorCenterGrid, sourcesVectorXGrid,
            sourcesVectorZGrid, sourcesVectorXZGrid, receiversVectorCenterGrid, receiversVectorXGrid,
            receiversVectorZGrid, receiversVectorXZGrid)

    def __str__(self):
        return " BornOp "

    def forward(self, add, model, data):
        with pyElastic_iso_float_nl.ostream_redirect():
            self.pyOp.forward(add, _cpp(model), _cpp(data))

    def adjoint(self, add, model, data):
        with pyElastic_iso_float_nl.ostream_redirect():
            self.pyOp.adjoint(add, _cpp(model), _cpp(data))

    def setBackground(self, elasticParam):
        with pyElastic_iso_float_nl.ostream_redirect():
            self.pyOp.setBackground(_cpp(elasticParam))
