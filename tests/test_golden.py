"""The oracle pinned against golden vectors produced by the reference's own
CUDA drivers (tests/golden/make_golden.py): same regular-grid inputs, outputs
compared within FP32 / FP64 round-off (the reference contracts to FMA on the
GPU, the oracle does not on the CPU)."""
import os

import numpy as np
import pytest

from oracle import oracle as O

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TOL = {"f": 1e-5, "d": 1e-12}


def load(prec):
    path = os.path.join(HERE, "ref_small_%s.npz" % prec)
    if not os.path.exists(path):
        pytest.fail("golden fixture missing: %s (generate with tests/golden/make_golden.py on a GPU)" % path)
    z = np.load(path)
    g = {k[2:]: z[k].item() for k in z.files if k.startswith("g_")}
    L = lambda name, n: [z["%s_%d" % (name, i)] for i in range(n)]  # noqa: E731
    return z, g, L


def rel(a, b):
    return O.rel_l2(np.concatenate([x.ravel() for x in a]), np.concatenate([x.ravel() for x in b]))


@pytest.mark.parametrize("prec", ["f", "d"])
def test_oracle_matches_reference_gpu(prec):
    z, g, L = load(prec)
    orc = O.Oracle(prec)
    med, model, data, fine, dm = L("med", 5), L("model", 5), L("data", 5), L("fine", 5), L("dm", 5)
    sp, rp = L("sp", 4), L("rp", 4)
    d = [np.zeros_like(a) for a in data]
    orc.nl_prop(0, g, med, [a.copy() for a in model], d, sp, rp)
    assert rel(d, L("out_nl_fwd_data", 5)) < TOL[prec]
    m = [np.zeros_like(a) for a in model]
    orc.nl_prop(1, g, med, m, [a.copy() for a in data], sp, rp)
    assert rel(m, L("out_nl_adj_model", 5)) < TOL[prec]
    d = [np.zeros_like(a) for a in data]
    orc.born_prop(0, g, med, fine, [a.copy() for a in dm], d, sp, rp)
    assert rel(d, L("out_born_fwd_data", 5)) < TOL[prec]
    m = [a.copy() for a in dm]
    orc.born_prop(1, g, med, fine, m, [a.copy() for a in data], sp, rp)
    assert rel(m, L("out_born_adj_dm", 5)) < TOL[prec]
    # the outputs are not trivially zero
    assert max(np.abs(a).max() for a in L("out_nl_fwd_data", 5)) > 0
    assert max(np.abs(a).max() for a in L("out_born_fwd_data", 5)) > 0
