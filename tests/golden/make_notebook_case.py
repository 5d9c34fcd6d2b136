"""Generates tests/golden/notebook_layers.npz from the reference's own notebook
inputs: the layered VpVsRho models notebooks/true_layers.H and
notebooks/smooth_layers.H (SEP headers + big-endian xdr_float binaries, read
here with the product's own sepio.readSep) and the parameter file
notebooks/EFWI_test.p (read with sepvec.paramObj).  The reference tree is
taken from EIO_REFERENCE_TREE (default: the reference checkout of this
machine).  Run from the repo root:

    python tests/golden/make_notebook_case.py

The fixture holds the two models [3][nx][nz] (vp, vs, rho), their axes and
the parameter file as key/value pairs, so that the tests that use the case run
where the reference tree is absent.
"""
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from elastic_isotropic_operators_b200 import sepio  # noqa: E402
from elastic_isotropic_operators_b200.sepvec import paramObj  # noqa: E402

TREE = os.environ.get("EIO_REFERENCE_TREE", "/root/reference/elastic_iso_lib")
OUT = os.path.join(ROOT, "tests", "golden", "notebook_layers.npz")


def read_case(tree=TREE):
    nb = os.path.join(tree, "notebooks")
    out = {}
    for name in ("true_layers", "smooth_layers"):
        v = sepio.readSep(os.path.join(nb, name + ".H"))
        out[name] = np.ascontiguousarray(v.getNdArray(), np.float32)
        out[name + "_axes"] = np.array([[a.n, a.o, a.d] for a in v.getHyper().axes], np.float64)
    par = paramObj.from_file(os.path.join(nb, "EFWI_test.p")).as_dict()
    out["par"] = np.array(json.dumps(par, sort_keys=True))
    return out


def main():
    np.savez_compressed(OUT, **read_case())
    print("wrote", OUT)


if __name__ == "__main__":
    main()
