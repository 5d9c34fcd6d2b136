"""Shot-parallel host logic on CPU: shot partitioning, the adjoint's model
stacking (all-reduce) and data gathering, run as two gloo ranks.

Each rank's local operator is the oracle's Born operator over its own block of
shots, so the test checks the exchange end to end against the serial oracle
over every shot without a GPU."""
import os
import socket

import numpy as np
import pytest

from elastic_isotropic_operators_b200.shots import ShotParallel, gather_data, local_vectors, shot_partition


@pytest.mark.parametrize("world", [1, 2, 3, 4, 7, 8])
@pytest.mark.parametrize("nExp", [0, 1, 2, 3, 10, 11, 64])
def test_shot_partition_covers_every_shot_once(nExp, world):
    blocks = [shot_partition(nExp, world, r) for r in range(world)]
    flat = [e for b in blocks for e in b]
    assert flat == list(range(nExp))
    sizes = [len(b) for b in blocks]
    assert max(sizes) - min(sizes) <= 1
    assert sizes == sorted(sizes, reverse=True)


def test_shot_partition_rejects_bad_requests():
    with pytest.raises(ValueError):
        shot_partition(4, 0, 0)
    with pytest.raises(ValueError):
        shot_partition(4, 2, 2)


def test_local_vectors_keeps_shared_entries():
    assert local_vectors(["a"], range(1, 3)) == ["a"]
    assert local_vectors(["a", "b", "c"], range(1, 3)) == ["b", "c"]


class _OracleBorn:
    """Test-only local operator: the oracle's Born operator over a subset of shots."""

    def __init__(self, w, shots):
        from oracle import oracle as O
        self.O = O
        self.orc = O.Oracle("f")
        c = O.Case.from_workload(w)
        c.src = [c.src[e] for e in shots]
        self.c = c
        self.sig = [w.source_signal()]

    def forward(self, add, model, data):
        d = self.O.born_forward(self.orc, self.c, model, self.sig)
        data[...] = d + (data if add else 0)

    def adjoint(self, add, model, data):
        m = self.O.born_adjoint(self.orc, self.c, data, self.sig)
        model[...] = m + (model if add else 0)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out_dir):
    import datetime
    import torch.distributed as dist
    from elastic_isotropic_operators_b200 import synthetic
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        w = synthetic.small(nshots=3, nts=60)
        op = ShotParallel(lambda shots: _OracleBorn(w, shots), w.nExp)
        rng = np.random.default_rng(5)
        model = (rng.standard_normal((3, w.nx, w.nz)) * 1e-2).astype(np.float32)
        data_all = rng.standard_normal((w.nExp, 5, len(w.rec_z), w.nts)).astype(np.float32)
        local = np.zeros((len(op.shots), 5, len(w.rec_z), w.nts), np.float32)
        op.forward(False, model, local)
        full = gather_data(local, w.nExp)
        grad = np.zeros_like(model)
        op.adjoint(False, grad, data_all[op.shots.start:op.shots.stop])
        np.savez(os.path.join(out_dir, "rank%d.npz" % rank), full=full, grad=grad,
                 shots=np.array(list(op.shots), np.int64))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_match_serial_oracle(tmp_path):
    import torch.multiprocessing as mp
    from oracle import oracle as O
    from elastic_isotropic_operators_b200 import synthetic
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    w = synthetic.small(nshots=3, nts=60)
    rng = np.random.default_rng(5)
    model = (rng.standard_normal((3, w.nx, w.nz)) * 1e-2).astype(np.float32)
    data_all = rng.standard_normal((w.nExp, 5, len(w.rec_z), w.nts)).astype(np.float32)
    orc = O.Oracle("f")
    c = O.Case.from_workload(w)
    sig = [w.source_signal()]
    want_data = O.born_forward(orc, c, model, sig)
    want_grad = O.born_adjoint(orc, c, data_all, sig)
    res = [np.load(tmp_path / ("rank%d.npz" % r)) for r in range(world)]
    assert list(res[0]["shots"]) == [0, 1] and list(res[1]["shots"]) == [2]
    for r in res:
        # every shot is computed by exactly one rank with the serial code: bitwise
        assert np.array_equal(r["full"], want_data)
        # the stacked model differs from the serial sum only by summation order
        assert O.rel_l2(r["grad"], want_grad) < 1e-6
    assert np.array_equal(res[0]["grad"], res[1]["grad"])


class _FakeGradient:
    """Test-only local operator: shot e contributes misfit 0.1 * (e + 1) and
    gradient (e + 1) * ones to the sum over its block."""

    def __init__(self, shots, shape):
        self.shots, self.shape = list(shots), shape

    def fwiGradient(self, model, sources, dObs, components=None):
        assert dObs.shape[0] == len(self.shots)
        w = sum(e + 1 for e in self.shots)
        return 0.1 * w, np.full(self.shape, float(w), np.float32)


def _rank_fwi(rank, world, port, out_dir):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        nExp, shape = 5, (3, 4, 6)
        op = ShotParallel(lambda shots: _FakeGradient(shots, shape), nExp)
        d_obs = np.zeros((len(op.shots), 2, 3, 7), np.float32)
        phi, g = op.fwiGradient(None, None, d_obs, shape=shape)
        np.savez(os.path.join(out_dir, "fwi%d.npz" % rank), phi=phi, g=g)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_shot_parallel_fwi_gradient_sums_over_ranks(tmp_path, world):
    import torch.multiprocessing as mp
    mp.start_processes(_rank_fwi, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    want = sum(e + 1 for e in range(5))
    res = [np.load(tmp_path / ("fwi%d.npz" % r)) for r in range(world)]
    for r in res:
        assert abs(float(r["phi"]) - 0.1 * want) < 1e-12
        assert np.array_equal(r["g"], np.full((3, 4, 6), float(want), np.float32))
    assert all(float(r["phi"]) == float(res[0]["phi"]) for r in res)


def _rank_fwi_no_shape(rank, world, port, out_dir):
    import datetime
    import time
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # one shot, three ranks: ranks 1 and 2 own none, and neither a model nor a shape is given
        op = ShotParallel(lambda shots: _FakeGradient(shots, (3, 4, 6)), 1)
        d_obs = np.zeros((len(op.shots), 2, 3, 7), np.float32)
        t0 = time.monotonic()
        try:
            op.fwiGradient(None, None, d_obs)
            outcome = "returned"
        except ValueError as ex:
            outcome = "ValueError: %s" % ex
        except RuntimeError as ex:
            outcome = "RuntimeError: %s" % ex
        np.savez(os.path.join(out_dir, "nf%d.npz" % rank), outcome=outcome, dt=time.monotonic() - t0)
    finally:
        dist.destroy_process_group()


def test_shot_parallel_fwi_gradient_fails_fast_on_every_rank(tmp_path):
    """A rank without shots and without a shape cannot form its part of the
    sum: every rank must raise (the owner of the shot included), well before
    the process group's timeout, instead of the owner waiting in the
    all-reduce."""
    import torch.multiprocessing as mp
    world = 3
    mp.start_processes(_rank_fwi_no_shape, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    res = [np.load(tmp_path / ("nf%d.npz" % r)) for r in range(world)]
    assert str(res[0]["outcome"]).startswith("RuntimeError"), str(res[0]["outcome"])
    for r in res[1:]:
        assert str(r["outcome"]).startswith("ValueError"), str(r["outcome"])
    assert all(float(r["dt"]) < 30.0 for r in res)


def _rank_fwi_model_shape(rank, world, port, out_dir):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        shape = (3, 4, 6)
        op = ShotParallel(lambda shots: _FakeGradient(shots, shape), 1)
        d_obs = np.zeros((len(op.shots), 2, 3, 7), np.float32)
        phi, g = op.fwiGradient(np.zeros(shape, np.float32), None, d_obs)
        np.savez(os.path.join(out_dir, "ms%d.npz" % rank), phi=phi, g=g)
    finally:
        dist.destroy_process_group()


def test_shot_parallel_fwi_gradient_shape_from_model(tmp_path):
    """Without ``shape`` the gradient takes the model's shape on every rank,
    so ranks without shots still join the sum."""
    import torch.multiprocessing as mp
    world = 3
    mp.start_processes(_rank_fwi_model_shape, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    for r in range(world):
        res = np.load(tmp_path / ("ms%d.npz" % r))
        assert abs(float(res["phi"]) - 0.1) < 1e-12
        assert np.array_equal(res["g"], np.ones((3, 4, 6), np.float32))
