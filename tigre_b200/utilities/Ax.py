"""tigre.Ax drop-in (Python/tigre/utilities/Ax.py:29-59 + _Ax.pyx:32-101).

numpy in -> numpy out through the host-pointer C entry points
(tigre_siddon_ray_projection / tigre_interpolation_projection); a CUDA torch
tensor in -> CUDA tensor out through the device-resident projector.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from .. import _native as N
from .gpu import device_list


def _is_cuda_tensor(x):
    return type(x).__module__.startswith("torch") and getattr(x, "is_cuda", False)


def Ax(img, geo, angles, projection_type="Siddon", **kwargs):  # noqa: N802
    if _is_cuda_tensor(img):
        from .. import projectors
        geox = N.checked_geometry(geo, angles)
        if tuple(img.shape) != tuple(int(v) for v in geox.nVoxel):
            raise ValueError("Input data should be of shape geo.nVoxel: %s not:%s" % (geox.nVoxel, tuple(img.shape)))
        plan = N.get_plan(geox, img.device.index)
        return projectors.ax(img.contiguous(), plan, _projector_name(projection_type))
    if img.dtype != np.float32:
        raise TypeError("Input data should be float32, not " + str(img.dtype))
    # the reference's np.isreal(img).all() check follows here (Ax.py:32-33); after the float32
    # test it is always true and costs a full pass over the volume, so it is omitted
    if any(np.asarray(img.shape) != np.asarray(geo.nVoxel)):
        raise ValueError("Input data should be of shape geo.nVoxel: " + str(geo.nVoxel) + " not:" + str(img.shape))
    geox = N.checked_geometry(geo, angles)
    devices = device_list(kwargs.get("gpuids", None))
    return _ax_host(img, geox, projection_type, geox.mode, devices)


def _projector_name(projection_type):
    if projection_type in ("Siddon", "ray-voxel"):
        return "Siddon"
    if projection_type == "interpolated":
        return "interpolated"
    print("Warning: Unknown projection_type, using default Siddon")
    return "Siddon"


def _ax_host(img, geox, projection_type, mode, devices):
    ptype = _projector_name(projection_type)
    angles = np.ascontiguousarray(np.asarray(geox.angles, dtype=np.float32).reshape(-1, 3))
    n = angles.shape[0]
    nv, nu = int(geox.nDetector[0]), int(geox.nDetector[1])
    out = N.host_empty((n, nv, nu))
    rows = (C.c_void_p * n)(*[out.ctypes.data + i * nv * nu * 4 for i in range(n)])
    cg = N.CGeometry(geox, n)
    ids = (C.c_int * len(devices))(*devices)
    img = np.ascontiguousarray(img)
    L = N.lib()
    if mode == "parallel":
        fn = L.tigre_interpolation_projection_parallel if ptype == "interpolated" else \
            L.tigre_siddon_ray_projection_parallel
    else:
        fn = L.tigre_interpolation_projection if ptype == "interpolated" else L.tigre_siddon_ray_projection
    rc = fn(img.ctypes.data, C.byref(cg.s), C.cast(rows, C.c_void_p), angles.ctypes.data, n, C.cast(ids, C.c_void_p),
            len(devices))
    if rc:
        raise ValueError("TIGRE: Call to Ax failed (code %d: %s)" % (rc, N.last_error()))
    return out
