"""CUDA-graph time loops (opt-in, eio_ctx_set_graphs): a replayed graph gives the same traces and images as
direct launches, reads the current contents of its buffers (new source traces,
new perturbation) rather than the ones it was captured with, and a new point
count captures a new graph.  Bitwise comparisons: the graph replays the same
kernels with the same arguments."""
import ctypes

import numpy as np
import pytest

from elastic_isotropic_operators_b200 import _lib, synthetic
from oracle import oracle as O

from helpers import Ctx, reg_inputs, rel

pytestmark = pytest.mark.gpu


def _copy(xs):
    return [x.copy() for x in xs]


def _all(c, r):
    out = {}
    for adj in (0, 1):
        pm, pd = c.nl(adj, _copy(r["model"]), _copy(r["data"]), r["sp"], r["rp"])
        out[("nl", adj)] = pm if adj else pd
        pdm, pd = c.born(adj, _copy(r["fine"]), _copy(r["dm"]), _copy(r["data"]), r["sp"], r["rp"])
        out[("born", adj)] = pdm if adj else pd
    return out


def _same(a, b):
    return all(np.array_equal(x, y) for x, y in zip(a, b))


@pytest.mark.parametrize("kind", [3, 5])
def test_graph_replay_equals_direct_launches(kind):
    w = synthetic.small(nts=60)
    r = reg_inputs(w, "f", seed=31)
    res = {}
    for graphs in (0, 1):
        c = Ctx(w)
        try:
            c.set_kernel(kind, 64, 16, 0)
            _lib.check(c.L.eio_ctx_set_graphs(c.h, graphs))
            first = _all(c, r)      # captures (graphs on)
            second = _all(c, r)     # replays
            for k in first:
                assert _same(first[k], second[k]), (graphs, k)
            res[graphs] = first
        finally:
            c.close()
    for k in res[0]:
        assert _same(res[0][k], res[1][k]), k


def test_graph_replay_reads_new_inputs_and_recaptures_on_new_geometry():
    w = synthetic.small(nts=60)
    c = Ctx(w)
    try:
        c.set_kernel(3, 64, 16, 0)
        _lib.check(c.L.eio_ctx_set_graphs(c.h, 1))
        for seed in (41, 42):            # same geometry, new traces and perturbation: replay
            r = reg_inputs(w, "f", seed=seed)
            got = _all(c, r)
            orc = r["orc"]
            for adj in (0, 1):
                m, d = _copy(r["model"]), _copy(r["data"])
                orc.nl_prop(adj, r["g"], r["med"], m, d, r["sp"], r["rp"])
                assert rel(got[("nl", adj)], m if adj else d) < 1e-5
                dm, d = _copy(r["dm"]), _copy(r["data"])
                orc.born_prop(adj, r["g"], r["med"], r["fine"], dm, d, r["sp"], r["rp"])
                assert rel(got[("born", adj)], dm if adj else d) < 1e-5
        # fewer receivers: other point counts, a new graph
        r = reg_inputs(w, "f", seed=43)
        r["rp"] = [p[: len(p) // 2] for p in r["rp"]]
        r["data"] = [d[: len(r["rp"][O.FIELD_GRID[f]])].copy() for f, d in enumerate(r["data"])]
        got = _all(c, r)
        orc = r["orc"]
        m, d = _copy(r["model"]), _copy(r["data"])
        orc.nl_prop(0, r["g"], r["med"], m, d, r["sp"], r["rp"])
        assert rel(got[("nl", 0)], d) < 1e-5
    finally:
        c.close()


def test_graph_stats_count_every_launch():
    """Launch counters and sampled timing also cover replayed graphs."""
    w = synthetic.small(nts=60)
    r = reg_inputs(w, "f", seed=47)
    c = Ctx(w)
    try:
        c.set_kernel(3, 64, 16, 0)
        _lib.check(c.L.eio_ctx_set_graphs(c.h, 1))
        c.nl(0, _copy(r["model"]), _copy(r["data"]), r["sp"], r["rp"])   # capture
        n = []
        for _ in range(2):
            _lib.check(c.L.eio_ctx_stats(c.h, 1, 1, None, None, None))
            c.nl(0, _copy(r["model"]), _copy(r["data"]), r["sp"], r["rp"])
            la, sl, ms = ctypes.c_longlong(), ctypes.c_longlong(), ctypes.c_double()
            _lib.check(c.L.eio_ctx_stats(c.h, 0, 1, ctypes.byref(la), ctypes.byref(sl), ctypes.byref(ms)))
            n.append((sl.value, ms.value))
        steps = (w.nts - 1) * 2
        for sl, ms in n:
            assert sl == steps and ms > 0, n
    finally:
        c.close()
