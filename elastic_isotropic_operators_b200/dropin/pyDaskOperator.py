"""``pyDaskOperator``: Dask clusters are not supported by this engine -- its
multi-GPU path is one process per GPU under torch.distributed
(elastic_isotropic_operators_b200.shots.ShotParallel).  The module exists so
that scripts importing it load; building a Dask operator raises."""


def _unsupported(*a, **k):
    raise NotImplementedError("Dask operators are not supported: run one process per GPU with torch.distributed "
                              "(elastic_isotropic_operators_b200.shots.ShotParallel)")


class DaskOperator:
    __init__ = _unsupported


class DaskSpreadOp:
    __init__ = _unsupported


class DaskCollectOp:
    __init__ = _unsupported


__all__ = ["DaskOperator", "DaskSpreadOp", "DaskCollectOp"]
