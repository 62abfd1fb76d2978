"""tigre.Atb drop-in (Python/tigre/utilities/Atb.py:9-40 + _Atb.pyx:31-90)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from .. import _native as N
from .errors import TigreCudaCallError
from .gpu import device_list


def _is_cuda_tensor(x):
    return type(x).__module__.startswith("torch") and getattr(x, "is_cuda", False)


def _backprojector_name(backprojection_type):
    if backprojection_type == "matched":
        return "matched"
    if backprojection_type == "FDK":
        return "FDK"
    print("Warning: Unknown backprojector, using default matched")
    return "matched"


def Atb(projections, geo, angles, backprojection_type="FDK", **kwargs):  # noqa: N802
    if _is_cuda_tensor(projections):
        from .. import projectors
        geox = N.checked_geometry(geo, angles)
        plan = N.get_plan(geox, projections.device.index)
        return projectors.atb(projections.contiguous(), plan, _backprojector_name(backprojection_type))
    if projections.dtype != np.float32:
        raise TypeError("Input data should be float32, not " + str(projections.dtype))
    # np.isreal(projections).all() (Atb.py:12-13) is always true for float32 and costs a full
    # pass over the projections: omitted
    geox = N.checked_geometry(geo, angles)
    want = (geox.angles.shape[0], int(geox.nDetector[0]), int(geox.nDetector[1]))
    if projections.shape != want:
        raise ValueError("Expected data shape: " + str(want) + " not compatible with: " + str(projections.shape))
    devices = device_list(kwargs.get("gpuids", None))
    return _atb_host(projections, geox, backprojection_type, geox.mode, devices)


def _atb_host(projections, geox, backprojection_type, mode, devices):
    btype = _backprojector_name(backprojection_type)
    angles = np.ascontiguousarray(np.asarray(geox.angles, dtype=np.float32).reshape(-1, 3))
    n = angles.shape[0]
    out = N.host_empty(tuple(int(v) for v in geox.nVoxel))
    cg = N.CGeometry(geox, n)
    ids = (C.c_int * len(devices))(*devices)
    proj = np.ascontiguousarray(projections)
    L = N.lib()
    if mode == "parallel":
        fn = L.tigre_voxel_backprojection_parallel
    else:
        fn = L.tigre_voxel_backprojection2 if btype == "matched" else L.tigre_voxel_backprojection
    rc = fn(proj.ctypes.data, C.byref(cg.s), out.ctypes.data, angles.ctypes.data, n, C.cast(ids, C.c_void_p),
            len(devices))
    if rc:
        raise TigreCudaCallError("Atb:", rc, N.last_error())
    return out
