"""TV denoising, drop-in for tigre.utilities.im3ddenoise (Python/tigre/utilities/
im_3d_denoise.py:7-27 over _tv_proximal.pyx:39-70): the volume is scaled to [0, 1], denoised
by the primal-dual ROF iteration of tv_proximal.cu (tigre_tvdenoising / tigre_tv_denoise,
unit spacing as the reference passes) and scaled back.  numpy in -> numpy out through the
host entry point; a CUDA tensor stays on the device."""
from __future__ import annotations

import ctypes as C

import numpy as np

from .. import _native as N
from .errors import TigreCudaCallError
from .gpu import device_list


def _tvdenoise_host(img, niter, lmbda, gpuids):
    src = np.ascontiguousarray(img, dtype=np.float32)
    out = np.empty_like(src)
    size = (C.c_long * 3)(src.shape[2], src.shape[1], src.shape[0])
    spacing = (C.c_float * 3)(1.0, 1.0, 1.0)
    devices = device_list(gpuids)
    ids = (C.c_int * len(devices))(*devices)
    rc = N.lib().tigre_tvdenoising(src.ctypes.data, out.ctypes.data, float(lmbda), C.cast(spacing, C.c_void_p),
                                   C.cast(size, C.c_void_p), int(niter), C.cast(ids, C.c_void_p), len(devices))
    if rc:
        raise TigreCudaCallError("tvdenoising:", rc, N.last_error())
    return out


def tv_denoise_device(img, niter, lmbda, work=None):
    """Device TV denoising of a float32 CUDA volume (nZ, nY, nX), unit spacing, no scaling."""
    import torch
    from ..projectors import _stream
    if img.dim() != 3 or not img.is_cuda or img.dtype != torch.float32:
        raise ValueError("expected a float32 CUDA volume (nZ, nY, nX)")
    x = img.contiguous()
    nz, ny, nx = x.shape
    L = N.lib()
    need = int(L.tigre_tv_denoise_work_floats(nx, ny, nz))
    if work is None or work.numel() < need:
        work = torch.empty(need, dtype=torch.float32, device=x.device)
    out = torch.empty_like(x)
    spacing = (C.c_float * 3)(1.0, 1.0, 1.0)
    N.check(L.tigre_tv_denoise(C.c_void_p(x.data_ptr()), C.c_void_p(out.data_ptr()), nx, ny, nz, float(lmbda),
                               C.cast(spacing, C.c_void_p), int(niter), C.c_void_p(work.data_ptr()), _stream(x)),
            "tigre_tv_denoise")
    return out


def im3ddenoise(img, iter=50, lmbda=15.0, gpuids=None):  # noqa: A002
    if img.ndim != 3:
        raise ValueError("Expected a 3D array (nZ, nY, nX), got shape %s." % (tuple(img.shape),))
    if type(img).__module__.startswith("torch") and getattr(img, "is_cuda", False):
        x = img.detach().float()
        imgmin = x.min()
        x = x - imgmin
        imgmax = x.max()
        x = x / imgmax
        x = tv_denoise_device(x, iter, lmbda)
        return x * imgmax + imgmin
    imgmin = np.amin(img.ravel())
    img = img - imgmin
    imgmax = np.amax(img.ravel())
    img = img / imgmax
    img = _tvdenoise_host(img, iter, lmbda, gpuids)
    img *= imgmax
    img += imgmin
    return img


im3DDenoise = im3ddenoise  # noqa: N816
