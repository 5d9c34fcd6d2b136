"""Source-wavefield checkpoints stored as 16-bit codes with a scale per
snapshot and field (BF16, FP16) for the Born operators: error against the FP64
oracle (elastic_iso_double semantics) and adjointness.

Both Born directions read the same quantized history, so forward and adjoint
stay exact adjoints of each other; the quantization only perturbs the
background wavefield they linearise around."""
import numpy as np
import pytest

from elastic_isotropic_operators_b200 import prop, synthetic
from oracle import oracle as O

pytestmark = pytest.mark.gpu

# relative L2 error against the FP64 oracle measured on this case on a B200
# (forward / gradient): FP32 8.2e-7 / 5.5e-7, FP16 1.8e-4 / 2.3e-5,
# BF16 1.3e-3 / 1.9e-4; the bounds keep a margin
BOUND = {0: 1e-4, 1: 5e-2, 2: 5e-3}


def _born(w, mode):
    src, rec = w.geometry()
    sig = [w.source_signal()]
    born = prop.BornElasticShotsGpu(w.elastic, w.par, sig, *src, *rec)
    born.setCheckpointPrecision(mode)
    return born, sig


@pytest.mark.parametrize("mode", [0, 1, 2])
def test_born_with_16bit_snapshots_vs_fp64_oracle(mode):
    w = synthetic.small()
    born, sig = _born(w, mode)
    c = O.Case.from_workload(w)
    dm = born.modelSpace()
    dm.getNdArray()[...] = w.extra["dmodel"]
    data = born.dataSpace()
    born.forward(False, dm, data)
    e_fwd = O.rel_l2(data.getNdArray(), O.born_forward(O.Oracle("d"), c, dm.getNdArray(), sig))
    g = born.modelSpace()
    born.adjoint(False, g, data)
    e_adj = O.rel_l2(g.getNdArray(), O.born_adjoint(O.Oracle("d"), c, data.getNdArray(), sig))
    print("checkpoint mode %d: Born forward rel L2 vs FP64 %.3e, adjoint (gradient) %.3e" % (mode, e_fwd, e_adj))
    assert e_fwd < BOUND[mode] and e_adj < BOUND[mode]
    assert np.abs(data.getNdArray()).max() > 0


@pytest.mark.parametrize("mode", [1, 2])
def test_16bit_snapshots_keep_the_dot_product(mode):
    w = synthetic.small()
    born, _ = _born(w, mode)
    assert born.dotTest(False, 1e-5), born.lastDotTest


def test_16bit_snapshots_need_sub_1():
    w = synthetic.small(nts=60, sub=2)
    born, _ = _born(w, 1)
    dm = born.modelSpace()
    dm.getNdArray()[...] = w.extra["dmodel"]
    with pytest.raises(prop.EioError) as ei:
        born.forward(False, dm, born.dataSpace())
    assert ei.value.code == -5
