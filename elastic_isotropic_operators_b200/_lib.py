"""ctypes binding of the C ABI declared in include/eio_b200.h.

The shared library is built in-tree (``libeio_b200.so`` next to this file).
There is no fallback: if the library is missing or a CUDA device cannot be
used, every operator raises instead of computing anything on the CPU.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libeio_b200.so")

EIO_OK = 0
_ERRORS = {
    -1: "invalid argument",
    -2: "finite-difference QC failed",
    -3: "CUDA error",
    -4: "acquisition device out of bounds",
    -5: "unsupported option",
    -6: "out of memory",
    -7: "device wait timed out",
    -8: "non-finite output",
}

F = ctypes.c_float
I = ctypes.c_int
P = ctypes.c_void_p
FP = ctypes.POINTER(ctypes.c_float)
IP = ctypes.POINTER(ctypes.c_int)


class EioError(RuntimeError):
    """Raised for every non-zero status returned by the C ABI."""

    def __init__(self, code, msg):
        super().__init__("%s (%d): %s" % (_ERRORS.get(code, "error"), code, msg))
        self.code = code


class FdParams(ctypes.Structure):
    """Mirror of ``eio_fd_params`` (the par-file keys of fdParamElastic)."""

    _fields_ = [
        ("nts", I), ("dts", F), ("ots", F), ("sub", I),
        ("nz", I), ("nx", I), ("oz", F), ("ox", F), ("dz", F), ("dx", F),
        ("zPadMinus", I), ("zPadPlus", I), ("xPadMinus", I), ("xPadPlus", I),
        ("fMax", F), ("blockSize", I), ("fat", I), ("alphaCos", F),
        ("surfaceCondition", I), ("mod_par", I), ("errorTolerance", F),
    ]


_lib = None

# name -> (restype, argtypes)
_SIGS = {
    "eio_fd_params_default": (None, [ctypes.POINTER(FdParams)]),
    "eio_last_error": (ctypes.c_char_p, []),
    "eio_version": (I, []),
    "eio_sinterp_create": (I, [FP, FP, I, I, F, F, I, F, F, I, ctypes.c_char_p, I, I, F, F, ctypes.POINTER(P)]),
    "eio_sinterp_destroy": (None, [P]),
    "eio_sinterp_sizes": (I, [P, IP, IP, IP]),
    "eio_sinterp_positions": (I, [P, IP]),
    "eio_sinterp_weights": (I, [P, IP, FP]),
    "eio_sinterp_forward": (I, [P, I, FP, FP]),
    "eio_sinterp_adjoint": (I, [P, I, FP, FP]),
    "eio_medium_prepare": (I, [ctypes.POINTER(FdParams), FP, FP, FP, FP, FP, FP]),
    "eio_stagger": (I, [I, I, I, I, I, FP, FP]),
    "eio_time_interp": (I, [I, I, I, F, F, I, I, FP, FP]),
    "eio_ctx_create": (I, [ctypes.POINTER(FdParams), FP, I, ctypes.POINTER(P)]),
    "eio_ctx_set_background": (I, [P, FP]),
    "eio_ctx_destroy": (None, [P]),
    "eio_ctx_set_checkpoint_precision": (I, [P, I]),
    "eio_ctx_get_medium": (I, [P, FP, FP, FP, FP, FP]),
    "eio_ctx_counts": (I, [P, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong)]),
    "eio_ctx_stream": (P, [P]),
    "eio_ctx_set_kernel": (I, [P, I, I, I, I]),
    "eio_ctx_get_kernel": (I, [P, IP, IP, IP, IP]),
    "eio_ctx_autotune": (I, [P, IP, IP, IP, IP]),
    "eio_ctx_set_wait_limit": (I, [P, ctypes.c_longlong]),
    "eio_ctx_step_cells": (I, [P, ctypes.POINTER(ctypes.c_longlong)]),
    "eio_ctx_set_persistent": (I, [P, I]),
    "eio_ctx_set_born_batch": (I, [P, I]),
    "eio_ctx_get_persistent": (I, [P, IP]),
    "eio_ctx_get_wait_limit": (I, [P, ctypes.POINTER(ctypes.c_longlong)]),
    "eio_ctx_stats": (I, [P, I, I, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong),
                          ctypes.POINTER(ctypes.c_double)]),
    "eio_ctx_set_graphs": (I, [P, I]),
    "eio_ctx_set_shot_windows": (I, [P, I, IP, IP]),
    "eio_ctx_set_lanes": (I, [P, I]),
    "eio_ctx_set_shot_batch": (I, [P, I]),
    "eio_ctx_get_lanes": (I, [P, IP, IP]),
    "eio_born_shots_dev": (I, [P, I, I, P, P, P, P, IP, P, IP]),
    "eio_fwi_gradient": (I, [P, I, I, FP, FP, I, IP, P, P, I, P, FP, ctypes.POINTER(ctypes.c_double)]),
    "eio_reduce64": (I, [I, I, I, P, P, ctypes.c_longlong, I, ctypes.POINTER(ctypes.c_double)]),
    "eio_cnn_conv3x3": (I, [I, I, I, I, I, P, P, P, I, P, P, P]),
    "eio_cnn_set_conv_path": (I, [I]),
    "eio_cnn_get_conv_path": (I, [IP]),
    "eio_cnn_status": (I, [I, IP]),
    "eio_cnn_set_wait_limit": (I, [ctypes.c_longlong]),
    "eio_cnn_get_wait_limit": (I, [ctypes.POINTER(ctypes.c_longlong)]),
    "eio_cnn_wgrad_scratch": (I, [I, I, I, I, I, ctypes.POINTER(ctypes.c_longlong)]),
    "eio_cnn_conv3x3_wgrad": (I, [I, I, I, I, I, P, P, P, P, ctypes.c_longlong, P]),
    "eio_cnn_flip": (I, [I, I, P, P, P]),
    "eio_cnn_mse": (I, [ctypes.c_longlong, I, I, P, P, P, P, P, P]),
    "eio_cnn_adam": (I, [ctypes.c_longlong, P, P, P, P, F, F, F, F, I, P, P]),
    "eio_gemm_bf16": (I, [ctypes.c_longlong, ctypes.c_longlong, ctypes.c_longlong, P, ctypes.c_longlong, P,
                          ctypes.c_longlong, P, P, P, I, I, P, P]),
    "eio_gemm_set_wait_limit": (I, [ctypes.c_longlong]),
    "eio_gemm_status": (I, [I, P]),
    "eio_ctx_set_history_location": (I, [P, I]),
    "eio_ctx_get_history_location": (I, [P, P]),
    "eio_ctx_set_check_finite": (I, [P, I]),
    "eio_set_device_memory_cap": (I, [ctypes.c_longlong]),
    "eio_get_device_memory_used": (I, [P]),
    "eio_unet_set_tma": (I, [I]),
    "eio_unet_get_tma": (I, [P]),
    "eio_unet_conv3x3": (I, [I, I, I, I, I, P, P, P, P, I, P]),
    "eio_unet_wgrad_scratch": (I, [I, I, I, I, I, P]),
    "eio_unet_conv3x3_wgrad": (I, [I, I, I, I, I, P, P, P, P, ctypes.c_longlong, P]),
    "eio_unet_flip": (I, [I, I, P, P, P]),
    "eio_unet_resample": (I, [I, I, I, I, I, P, P, I, P]),
    "eio_unet_concat": (I, [I, ctypes.c_longlong, I, I, P, I, P, I, P, P]),
    "eio_unet_relu_adj": (I, [ctypes.c_longlong, P, P, P, I, P]),
    "eio_ctx_pair_stats": (I, [P, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_double)]),
    "eio_nl_fwd_reg": (I, [P, P, P, P, IP, P, IP]),
    "eio_nl_adj_reg": (I, [P, P, P, P, IP, P, IP]),
    "eio_born_fwd_reg": (I, [P, P, P, P, P, IP, P, IP]),
    "eio_born_adj_reg": (I, [P, P, P, P, P, IP, P, IP]),
    "eio_nl_fwd_reg_dev": (I, [P, P, P, P, IP, P, IP]),
    "eio_nl_adj_reg_dev": (I, [P, P, P, P, IP, P, IP]),
    "eio_born_fwd_reg_dev": (I, [P, P, P, P, P, IP, P, IP]),
    "eio_born_adj_reg_dev": (I, [P, P, P, P, P, IP, P, IP]),
    "eio_born_prepare_sources": (I, [P, FP, P, P]),
    "eio_born_prepare_model": (I, [P, FP, P]),
    "eio_nl_prepare_sources": (I, [P, FP, P, P]),
    "eio_nl_fwd_noalloc": (I, [ctypes.POINTER(FdParams), P, P, P, P, IP, P, IP, P]),
    "eio_nl_forward": (I, [P, I, I, I, FP, FP, P, P, I]),
    "eio_nl_forward_wavefield": (I, [P, I, I, I, FP, FP, P, P, I, I, FP]),
    "eio_nl_adjoint_wavefield": (I, [P, I, I, I, FP, FP, P, P, I, I, FP]),
    "eio_nl_adjoint": (I, [P, I, I, I, FP, FP, P, P, I]),
    "eio_born_forward": (I, [P, I, I, FP, FP, P, I, P, P, I]),
    "eio_born_adjoint": (I, [P, I, I, FP, FP, P, I, P, P, I]),
}


def exported_symbols():
    """Names of every entry point declared in include/eio_b200.h."""
    return sorted(_SIGS)


def lib():
    """Load (once) and return the shared library; raises if it was not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise EioError(-5, "libeio_b200.so not built (run __graft_entry__.build())")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(status):
    if status != EIO_OK:
        msg = lib().eio_last_error()
        raise EioError(status, msg.decode() if msg else "")


def fptr(a):
    """float* of a C-contiguous float32 numpy array (no copy)."""
    assert a.dtype == np.float32 and a.flags["C_CONTIGUOUS"], "need contiguous float32"
    return a.ctypes.data_as(FP)


def iptr(a):
    assert a.dtype == np.int32 and a.flags["C_CONTIGUOUS"], "need contiguous int32"
    return a.ctypes.data_as(IP)


def ptr_array(addrs, ctype=ctypes.c_void_p):
    """C array of raw pointers (keeps no references: callers hold the buffers)."""
    arr = (ctype * len(addrs))()
    for i, a in enumerate(addrs):
        arr[i] = a
    return arr


def addr(a):
    """Raw address of a numpy array or a torch tensor."""
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    return int(a.data_ptr())
