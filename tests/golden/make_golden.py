"""Generates the golden vectors of tests/golden/ by running the REFERENCE'S OWN
CUDA drivers (oracle/_ref: elastic_iso_float and elastic_iso_double built for
sm_100a from the reference tree) on small seeded regular-grid inputs prepared
by the oracle's restated host preparation.  Needs a GPU; run from the repo root:

    python tests/golden/make_golden.py

Writes ref_small_{f,d}.npz: inputs (grid, medium, positions, traces) and the
reference outputs of the nonlinear forward/adjoint and Born forward/adjoint.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

from elastic_isotropic_operators_b200 import synthetic  # noqa: E402
from oracle import oracle as O  # noqa: E402
from helpers import reg_inputs  # noqa: E402


def golden_case():
    return synthetic.small(nz=56, nx=72, nts=100, nshots=1, nrec=10, seed=21)


def main():
    w = golden_case()
    for prec in ("f", "d"):
        r = reg_inputs(w, prec, seed=31)
        ref = O.RefGpu(prec)
        out = {}
        m, d = [a.copy() for a in r["model"]], [np.zeros_like(a) for a in r["data"]]
        ref.nl_prop(0, r["g"], r["med"], m, d, r["sp"], r["rp"])
        out["nl_fwd_data"] = d
        m, d = [np.zeros_like(a) for a in r["model"]], [a.copy() for a in r["data"]]
        ref.nl_prop(1, r["g"], r["med"], m, d, r["sp"], r["rp"])
        out["nl_adj_model"] = m
        dm, d = [a.copy() for a in r["dm"]], [np.zeros_like(a) for a in r["data"]]
        ref.born_prop(0, r["g"], r["med"], r["fine"], dm, d, r["sp"], r["rp"])
        out["born_fwd_data"] = d
        dm, d = [a.copy() for a in r["dm"]], [a.copy() for a in r["data"]]
        ref.born_prop(1, r["g"], r["med"], r["fine"], dm, d, r["sp"], r["rp"])
        out["born_adj_dm"] = dm
        save = {}
        for k in ("nz", "nx", "dz", "dx", "nts", "dts", "S", "minPad", "alphaCos"):
            save["g_" + k] = np.array(r["g"][k])
        for name in ("med", "model", "data", "fine", "dm"):
            for i, a in enumerate(r[name]):
                save["%s_%d" % (name, i)] = a
        for i in range(4):
            save["sp_%d" % i] = r["sp"][i]
            save["rp_%d" % i] = r["rp"][i]
        for k, v in out.items():
            for i, a in enumerate(v):
                save["out_%s_%d" % (k, i)] = a
        path = os.path.join(ROOT, "tests", "golden", "ref_small_%s.npz" % prec)
        np.savez_compressed(path, **save)
        print("wrote", path)


if __name__ == "__main__":
    main()
