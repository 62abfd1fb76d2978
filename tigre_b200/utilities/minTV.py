"""POCS-TV denoiser, drop-in for the _minTV extension (_minTV.pyx:39-64)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from .. import _native as N
from .errors import TigreCudaCallError
from .gpu import device_list


def minTV(src, alpha=15.0, maxiter=100, gpuids=None):  # noqa: N802
    if type(src).__module__.startswith("torch") and getattr(src, "is_cuda", False):
        from .. import projectors
        out = src.detach().to(dtype=src.dtype).contiguous().clone()
        return projectors.tv_pocs_(out, float(alpha), int(maxiter))
    src = np.ascontiguousarray(src, dtype=np.float32)
    if src.ndim != 3:
        raise ValueError("minTV expects a 3-D volume")
    out = np.empty_like(src)
    size = (C.c_long * 3)(src.shape[2], src.shape[1], src.shape[0])
    devices = device_list(gpuids)
    ids = (C.c_int * len(devices))(*devices)
    rc = N.lib().tigre_pocs_tv(src.ctypes.data, out.ctypes.data, float(alpha), C.cast(size, C.c_void_p),
                               int(maxiter), C.cast(ids, C.c_void_p), len(devices))
    if rc:
        raise TigreCudaCallError("minimizeTV:POCS_TV:", rc, N.last_error())
    return out
