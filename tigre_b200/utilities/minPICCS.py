"""PICCS TV descent, drop-in for the _minPICCS extension (_minPICCS.pyx:39-64)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from .. import _native as N
from .errors import TigreCudaCallError
from .gpu import device_list


def minPICCS(src, prior, alpha=15.0, maxiter=100, ratio=0.95, gpuids=None):  # noqa: N802
    """maxiter steps of f -= alpha g/|g|, g = (1-ratio) grad TV(f) + ratio grad TV(f - prior).
    numpy in, numpy out; CUDA tensors stay on their device."""
    if type(src).__module__.startswith("torch") and getattr(src, "is_cuda", False):
        from .. import projectors
        out = src.detach().contiguous().clone()
        return projectors.tv_piccs_(out, prior.detach().contiguous(), float(alpha), float(ratio), int(maxiter))
    src = np.ascontiguousarray(src, dtype=np.float32)
    prior = np.ascontiguousarray(prior, dtype=np.float32)
    if src.ndim != 3 or prior.shape != src.shape:
        raise ValueError("minPICCS expects two 3-D volumes of the same size")
    out = np.empty_like(src)
    size = (C.c_long * 3)(src.shape[2], src.shape[1], src.shape[0])
    devices = device_list(gpuids)
    ids = (C.c_int * len(devices))(*devices)
    rc = N.lib().tigre_piccs_tv(src.ctypes.data, prior.ctypes.data, out.ctypes.data, float(alpha), float(ratio),
                                C.cast(size, C.c_void_p), int(maxiter), C.cast(ids, C.c_void_p), len(devices))
    if rc:
        raise TigreCudaCallError("minimizeTV:PICCS_TV:", rc, N.last_error())
    return out
