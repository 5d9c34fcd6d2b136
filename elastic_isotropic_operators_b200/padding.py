"""Model padding for the finite-difference grid (padElasticFileGpuMain,
seis_utils_float/src/padElasticFileGpuMain.cpp).

The engine needs (nz - 2*fat) and (nx - 2*fat) to be multiples of blockSize:
the model gets zPad / xPad damping cells on each side, the far pads grow
(zPadPlus, xPadPlus) to reach the next multiple, then a fat-cell frame goes
around everything.  Pad cells copy the nearest edge value of the model.  With
surfaceCondition = 1 the top pad is fat cells only, so the free surface at
z = 2*fat falls on the first model row.
"""
import math

import numpy as np

from .sepvec import axis, floatVector, hypercube

__all__ = ["pad_sizes", "pad_elastic_array", "padElasticFile"]


def pad_sizes(nz, nx, zPad, xPad, fat=4, blockSize=16, surfaceCondition=0):
    """(zPadMinus, zPadPlus, xPadMinus, xPadPlus) of the padded grid."""
    if surfaceCondition == 0:
        nzTotal = zPad * 2 + nz
        zMinus = zPad
    elif surfaceCondition == 1:
        nzTotal = zPad + nz + fat
        zMinus = fat
    else:
        raise ValueError("ERROR UNKNOWN SURFACE CONDITION PARAMETER")
    zPlus = int(math.ceil(float(nzTotal) / blockSize)) * blockSize - nz - zMinus
    nxTotal = xPad * 2 + nx
    xPlus = int(math.ceil(float(nxTotal) / blockSize)) * blockSize - nx - xPad
    return zMinus, zPlus, xPad, xPlus


def pad_elastic_array(ep, zPad, xPad, fat=4, blockSize=16, surfaceCondition=0):
    """ep [npar][nx][nz] -> padded [npar][nxNew][nzNew] and the pad sizes."""
    ep = np.asarray(ep, dtype=np.float32)
    if ep.ndim == 2:
        ep = ep[None]
    npar, nx, nz = ep.shape
    zMinus, zPlus, xMinus, xPlus = pad_sizes(nz, nx, zPad, xPad, fat, blockSize, surfaceCondition)
    nzN = zMinus + zPlus + nz + 2 * fat
    nxN = xMinus + xPlus + nx + 2 * fat
    out = np.zeros((npar, nxN, nzN), dtype=np.float32)
    z0, x0 = fat + zMinus, fat + xMinus
    out[:, x0:x0 + nx, z0:z0 + nz] = ep
    out[:, x0:x0 + nx, :z0] = ep[:, :, :1]
    out[:, x0:x0 + nx, z0 + nz:] = ep[:, :, -1:]
    out[:, :x0, :] = out[:, x0:x0 + 1, :]
    out[:, x0 + nx:, :] = out[:, x0 + nx - 1:x0 + nx, :]
    return out, dict(zPadMinus=zMinus, zPadPlus=zPlus, xPadMinus=xMinus, xPadPlus=xPlus)


def padElasticFile(model, zPad, xPad, fat=4, blockSize=16, surfaceCondition=0):
    """Pad a model vector (axes z, x[, parameter]) and shift its origins;
    returns the padded vector and the four pad sizes for the par file."""
    hyp = model.getHyper()
    az, ax = hyp.getAxis(1), hyp.getAxis(2)
    apar = hyp.getAxis(3) if hyp.getNdim() >= 3 else axis(1)
    arr = model.getNdArray().reshape(apar.n, ax.n, az.n)
    out, pads = pad_elastic_array(arr, zPad, xPad, fat, blockSize, surfaceCondition)
    oz = az.o - (fat + pads["zPadMinus"]) * az.d
    ox = ax.o - (fat + pads["xPadMinus"]) * ax.d
    h = hypercube(axes=[axis(out.shape[2], oz, az.d, az.label, az.unit),
                        axis(out.shape[1], ox, ax.d, ax.label, ax.unit),
                        axis(apar.n, apar.o, apar.d, apar.label, apar.unit)])
    return floatVector(h, out), pads
