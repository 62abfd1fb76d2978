"""Adaptive-weighted TV descent, drop-in for the _AwminTV extension (_AwminTV.pyx:33-64)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from .. import _native as N
from .gpu import device_list


def AwminTV(src, alpha=15.0, maxiter=100, delta=-0.005, gpuids=None):  # noqa: N802
    """maxiter steps of f -= alpha g/|g| with g the gradient of the adaptive-weighted TV
    (weights exp(-(d/delta)^2) on every difference).  numpy in, numpy out; a CUDA tensor stays
    on its device."""
    if type(src).__module__.startswith("torch") and getattr(src, "is_cuda", False):
        from .. import projectors
        out = src.detach().contiguous().clone()
        return projectors.tv_aw_pocs_(out, float(alpha), int(maxiter), float(delta))
    src = np.ascontiguousarray(src, dtype=np.float32)
    if src.ndim != 3:
        raise ValueError("AwminTV expects a 3-D volume")
    out = np.empty_like(src)
    size = (C.c_long * 3)(src.shape[2], src.shape[1], src.shape[0])
    devices = device_list(gpuids)
    ids = (C.c_int * len(devices))(*devices)
    rc = N.lib().tigre_aw_pocs_tv(src.ctypes.data, out.ctypes.data, float(alpha), C.cast(size, C.c_void_p),
                                  int(maxiter), float(delta), C.cast(ids, C.c_void_p), len(devices))
    if rc:
        # _AwminTV.pyx:31-33
        raise ValueError("TIGRE:Call to aw_pocs_tv failed: " + N.last_error())
    return out
