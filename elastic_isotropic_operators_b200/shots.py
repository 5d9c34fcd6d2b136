"""Shot-parallel execution: one process per GPU under torch.distributed.

The reference spreads the shots of one operator call over the GPUs of a single
process with an OpenMP loop, one thread per GPU and ``schedule(dynamic,1)``
(F/src/BornElasticShotsGpu.cpp:178-207 forward, :275-306 adjoint;
F/src/nonlinearPropElasticShotsGpu.cpp the same), writes each shot's data
slice straight into the shared data vector, and stacks the per-GPU model
slices of the adjoint on the host (BornElasticShotsGpu.cpp:312-323).

Here every rank owns a fixed contiguous block of shots (``shot_partition``),
runs them through its own single-GPU operator, and the stacking becomes one
all-reduce of the model vector over the process group (NCCL between GPUs,
gloo on CPU).  Shots are independent, so the forward needs no exchange at all;
``gather_data`` assembles the full data vector only when a caller asks for it.
"""
import numpy as np

__all__ = ["shot_partition", "local_vectors", "stack_model", "gather_data", "sum_in_rank_order", "all_ranks_ok",
           "ShotParallel"]


def shot_partition(nExp, world, rank):
    """Contiguous block of shot indices owned by ``rank``: the first
    ``nExp % world`` ranks take one shot more than the others."""
    if nExp < 0 or world < 1 or not 0 <= rank < world:
        raise ValueError("bad shot partition request (nExp=%d, world=%d, rank=%d)" % (nExp, world, rank))
    base, extra = divmod(nExp, world)
    start = rank * base + min(rank, extra)
    return range(start, start + base + (1 if rank < extra else 0))


def local_vectors(vectors, shots):
    """Per-shot list (length nExp) -> the entries of ``shots``; a list of length
    one (a geometry or signal shared by every shot) is kept as it is."""
    vectors = list(vectors)
    if len(vectors) == 1:
        return vectors
    return [vectors[e] for e in shots]


def _group_device(group):
    import torch
    import torch.distributed as dist
    if dist.get_backend(group) == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def stack_model(model, group=None):
    """Sum a model-space array (numpy, float32) over the ranks of ``group`` in
    place: the host stacking of the reference's per-GPU model slices."""
    import torch
    import torch.distributed as dist
    if not dist.is_initialized() or dist.get_world_size(group) == 1:
        return model
    dev = _group_device(group)
    t = torch.from_numpy(np.ascontiguousarray(model, np.float32)).to(dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    model[...] = t.cpu().numpy().reshape(model.shape)
    return model


def gather_data(local, nExp, group=None):
    """Assemble the full data vector [nExp][...] from each rank's block of
    shots [len(shot_partition)][...]; every rank receives the whole vector."""
    import torch
    import torch.distributed as dist
    if not dist.is_initialized() or dist.get_world_size(group) == 1:
        return np.array(local, np.float32, copy=True)
    world = dist.get_world_size(group)
    mine = dist.get_rank(group)
    dev = _group_device(group)
    cap = len(shot_partition(nExp, world, 0))        # the largest block
    shape = tuple(local.shape[1:])
    buf = torch.zeros((cap,) + shape, dtype=torch.float32, device=dev)
    n = len(shot_partition(nExp, world, mine))
    if n:
        buf[:n] = torch.from_numpy(np.ascontiguousarray(local, np.float32)).to(dev)
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf, group=group)
    out = np.zeros((nExp,) + shape, np.float32)
    for r in range(world):
        sh = shot_partition(nExp, world, r)
        if len(sh):
            out[sh.start:sh.stop] = parts[r][:len(sh)].cpu().numpy()
    return out


def sum_in_rank_order(value, group=None):
    """Sum of a float over the ranks of ``group``, added in rank order (FP64),
    so that every rank gets the same bits whatever the collective's order."""
    import torch
    import torch.distributed as dist
    if not dist.is_initialized() or dist.get_world_size(group) == 1:
        return float(value)
    dev = _group_device(group)
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    parts = [torch.empty_like(t) for _ in range(dist.get_world_size(group))]
    dist.all_gather(parts, t, group=group)
    total = 0.0
    for p in parts:
        total += float(p.item())
    return total


def all_ranks_ok(ok, group=None):
    """True on every rank when ``ok`` holds on every rank of ``group``: one
    all-reduce (MIN) of a flag, so that the ranks agree on an error before any
    of them enters a collective that a failed rank would never join."""
    import torch
    import torch.distributed as dist
    if not dist.is_initialized() or dist.get_world_size(group) == 1:
        return bool(ok)
    t = torch.tensor([1 if ok else 0], dtype=torch.int32, device=_group_device(group))
    dist.all_reduce(t, op=dist.ReduceOp.MIN, group=group)
    return bool(t.item())


class ShotParallel:
    """An operator over nExp shots split across the ranks of a process group.

    ``make_local(shots)`` builds this rank's operator over the shot indices
    ``shots`` (for instance ``BornElasticShotsGpu`` constructed with
    ``local_vectors`` of the geometry and signal lists); it is not called when
    the rank owns no shot.  ``forward``/``adjoint`` take this rank's data
    block [len(shots)][5][nRec][nts].  When ``stacked`` (Born model, or a
    nonlinear source signal shared by every shot) the adjoint's model is summed
    over the ranks; otherwise each rank keeps its own model block.
    """

    def __init__(self, make_local, nExp, group=None, stacked=True):
        import torch.distributed as dist
        self.group = group
        self.world = dist.get_world_size(group) if dist.is_initialized() else 1
        self.rank = dist.get_rank(group) if dist.is_initialized() else 0
        self.nExp = nExp
        self.shots = shot_partition(nExp, self.world, self.rank)
        self.stacked = stacked
        self.local = make_local(self.shots) if len(self.shots) else None

    def forward(self, add, model, data):
        if self.local is not None:
            self.local.forward(add, model, data)

    def fwiGradient(self, model, sources, dObs, components=None, shape=None):
        """FWI misfit and gradient over every rank's shots: this rank's local
        operator (a BornElasticShotsGpu) runs the fused gradient of its block
        (``sources`` and ``dObs`` are this rank's entries), the gradients are
        summed over the ranks (stack_model) and the misfits added in rank order.

        ``shape``: the gradient's shape; by default the shape of ``model``
        (the gradient lives in the elastic model's space).  Every rank resolves
        it and runs its own block before any collective; the ranks then agree
        on success (all_ranks_ok), so an error on one rank -- a missing shape on
        a rank without shots, a failed propagation -- raises on every rank
        instead of leaving the others waiting in the sum."""
        err = None
        phi, g = 0.0, None
        try:
            if shape is None and model is not None:
                m = model.getNdArray() if hasattr(model, "getNdArray") else model
                shape = np.shape(m)
            if self.local is not None:
                phi, g = self.local.fwiGradient(model, sources, dObs, components)
                g = np.ascontiguousarray(g, np.float32)
                if shape is not None and g.shape != tuple(shape):
                    raise ValueError("local gradient shape %s, expected %s" % (g.shape, tuple(shape)))
            elif shape is None:
                raise ValueError("a rank without shots needs the gradient shape (give model or shape)")
            else:
                g = np.zeros(shape, np.float32)
        except Exception as ex:   # re-raised below, after every rank knows
            err = ex
        if not all_ranks_ok(err is None, self.group):
            if err is not None:
                raise err
            raise RuntimeError("fwiGradient failed on another rank of the group")
        stack_model(g, self.group)
        return sum_in_rank_order(phi, self.group), g

    def adjoint(self, add, model, data):
        m = model.getNdArray() if hasattr(model, "getNdArray") else model
        part = np.zeros_like(m)
        if self.local is not None:
            self.local.adjoint(False, part, data)
        if self.stacked:
            stack_model(part, self.group)
        if add:
            m += part
        else:
            m[...] = part
