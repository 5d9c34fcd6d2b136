"""The two-step kernel (kind 5, k_pair): two fine steps per launch on the tile
widened by the stencil radius.

Checks, through the C ABI on cuda:0:
  * the single-step kernel (kind 3) and the two-step kernel give the same
    traces and images (relative L2 <= 1e-6: the same operations on the same
    values; only the order of several sources summed into one cell may differ);
  * with sources and receivers placed on and next to tile edges in z and x
    (the injections a CTA makes into the ring of cells its neighbours own),
    the two-step kernel matches the FP32 oracle (relative L2 <= 1e-5);
  * the Born operators' mixed schedules (the last coarse interval of the
    source wavefield and the first of the adjoint run as single steps).
"""
import numpy as np
import pytest

from elastic_isotropic_operators_b200 import synthetic
from oracle import oracle as O

from helpers import Ctx, reg_inputs, rel

pytestmark = pytest.mark.gpu

TOL32 = 1e-5
TOL_SAME = 1e-6
FAT, TZ, TX = 4, 64, 16


def _copy(xs):
    return [x.copy() for x in xs]


PAD = 12   # the absorbing band of synthetic.small (white-noise traces there grow without bound)


def _edge_cells(nz, nx, n, rng):
    """n distinct cells on or within 4 cells of a tile edge (z or x), outside
    the absorbing band."""
    lo = FAT + PAD
    zs = [z for k in range(0, (nz - 2 * FAT) // TZ + 1) for z in range(FAT + k * TZ - 4, FAT + k * TZ + 4)]
    xs = [x for k in range(0, (nx - 2 * FAT) // TX + 1) for x in range(FAT + k * TX - 4, FAT + k * TX + 4)]
    zs = [z for z in zs if lo <= z < nz - lo]
    xs = [x for x in xs if lo <= x < nx - lo]
    cells = set()
    while len(cells) < n:
        if zs and rng.random() < 0.5:
            iz, ix = rng.choice(zs), rng.integers(lo, nx - lo)
        else:
            iz, ix = rng.integers(lo, nz - lo), rng.choice(xs)
        cells.add(int(ix) * nz + int(iz))
    return np.array(sorted(cells), np.int32)


def _edge_inputs(w, seed, nsrc=24, nrec=40):
    r = reg_inputs(w, "f", seed=seed)
    rng = np.random.default_rng(seed + 1)
    sp = [_edge_cells(w.nz, w.nx, nsrc, rng) for _ in range(4)]
    rp = [_edge_cells(w.nz, w.nx, nrec, rng) for _ in range(4)]
    nts = r["g"]["nts"]
    r["sp"], r["rp"] = sp, rp
    r["model"] = [rng.standard_normal((len(sp[O.FIELD_GRID[f]]), nts)).astype(np.float32) for f in range(5)]
    r["data"] = [rng.standard_normal((len(rp[O.FIELD_GRID[f]]), nts)).astype(np.float32) for f in range(5)]
    ntw = r["fine"][0].shape[1]
    r["fine"] = [rng.standard_normal((len(sp[O.FIELD_GRID[f]]), ntw)).astype(np.float32) for f in range(5)]
    return r


def _run(kind, w, r):
    c = Ctx(w)
    try:
        c.set_kernel(kind, 64, 16, 0)
        out = {}
        # the C entry points write their outputs into the arrays they get
        for adj in (0, 1):
            pm, pd = c.nl(adj, _copy(r["model"]), _copy(r["data"]), r["sp"], r["rp"])
            out[("nl", adj)] = pm if adj else pd
            pdm, pd = c.born(adj, _copy(r["fine"]), _copy(r["dm"]), _copy(r["data"]), r["sp"], r["rp"])
            out[("born", adj)] = pdm if adj else pd
        return out
    finally:
        c.close()


def _oracle(r):
    orc = r["orc"]
    out = {}
    for adj in (0, 1):
        m, d = _copy(r["model"]), _copy(r["data"])
        orc.nl_prop(adj, r["g"], r["med"], m, d, r["sp"], r["rp"])
        out[("nl", adj)] = m if adj else d
        dm, d = _copy(r["dm"]), _copy(r["data"])
        orc.born_prop(adj, r["g"], r["med"], r["fine"], dm, d, r["sp"], r["rp"])
        out[("born", adj)] = dm if adj else d
    return out


@pytest.mark.parametrize("shape", [(72, 104, 60), (136, 120, 61), (104, 120, 40)],
                         ids=["one_tile_row", "two_tile_rows", "ragged"])
def test_pair_matches_single_step_and_oracle_at_tile_edges(shape):
    nz, nx, nts = shape
    w = synthetic.small(nz=nz, nx=nx, nts=nts)
    r = _edge_inputs(w, seed=nz + nts)
    single = _run(3, w, r)
    pair = _run(5, w, r)
    want = _oracle(r)
    for key in want:
        assert rel(pair[key], single[key]) < TOL_SAME, (key, rel(pair[key], single[key]))
        assert rel(pair[key], want[key]) < TOL32, (key, rel(pair[key], want[key]))
        assert max(np.abs(x).max() for x in pair[key]) > 0, key


def test_pair_with_default_geometry_matches_single_step():
    w = synthetic.small()
    r = reg_inputs(w, "f", seed=23)
    single = _run(3, w, r)
    pair = _run(5, w, r)
    for key in single:
        assert rel(pair[key], single[key]) < TOL_SAME, (key, rel(pair[key], single[key]))


@pytest.mark.parametrize("ckpt", [1, 2])
def test_pair_16bit_checkpoints_match_single_step(ckpt):
    """The warp maxima behind the snapshot scales come from the same cells in
    both kernels, so the quantized history and the images agree."""
    import ctypes
    w = synthetic.small(nts=60)
    r = reg_inputs(w, "f", seed=29)
    res = {}
    for kind in (3, 5):
        c = Ctx(w)
        try:
            c.set_kernel(kind, 64, 16, 0)
            from elastic_isotropic_operators_b200 import _lib
            _lib.check(c.L.eio_ctx_set_checkpoint_precision(c.h, ctypes.c_int(ckpt)))
            out = []
            for adj in (0, 1):
                pdm, pd = c.born(adj, _copy(r["fine"]), _copy(r["dm"]), _copy(r["data"]), r["sp"], r["rp"])
                out.append(pdm if adj else pd)
            res[kind] = out
        finally:
            c.close()
    for a, b in zip(res[3], res[5]):
        assert rel(b, a) < TOL_SAME, rel(b, a)
