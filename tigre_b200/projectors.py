"""Device-resident projector pair and TV on torch CUDA tensors.

These call the device API of libtigre_b200 (tigre_ax / tigre_atb /
tigre_tv_*) on the tensor's current CUDA stream; nothing crosses to the host.
Layouts follow TIGRE: volume (nZ, nY, nX), projections (nAngles, nV, nU).
Storage may be float32, bfloat16 or float16; arithmetic is FP32, geometry FP64.
"""
from __future__ import annotations

import ctypes as C

import torch

from . import _native as N

_DT = {torch.float32: N.F32, torch.bfloat16: N.BF16, torch.float16: N.F16}

PROJECTORS = {"Siddon": N.PROJ_SIDDON, "ray-voxel": N.PROJ_SIDDON, "interpolated": N.PROJ_INTERPOLATED}
BACKPROJECTORS = {"FDK": N.BACKPROJ_FDK, "matched": N.BACKPROJ_MATCHED}


def _dt(t: torch.Tensor) -> int:
    try:
        return _DT[t.dtype]
    except KeyError:
        raise TypeError("unsupported storage dtype %s (float32, bfloat16, float16)" % t.dtype)


def _stream(t: torch.Tensor):
    return C.c_void_p(torch.cuda.current_stream(t.device).cuda_stream)


def _require(t: torch.Tensor, shape, name):
    if not t.is_cuda:
        raise ValueError("%s must be a CUDA tensor" % name)
    if tuple(t.shape) != tuple(shape):
        raise ValueError("%s should be of shape %s, not %s" % (name, tuple(shape), tuple(t.shape)))
    if not t.is_contiguous():
        raise ValueError("%s must be contiguous" % name)


def _range(plan, angle_range):
    a0, a1 = (0, plan.n) if angle_range is None else (int(angle_range[0]), int(angle_range[1]))
    if not (0 <= a0 < a1 <= plan.n):
        raise ValueError("angle range %s outside [0, %d)" % ((a0, a1), plan.n))
    return a0, a1


def ax(vol: torch.Tensor, plan: "N.Plan", projection_type="Siddon", angle_range=None, out=None, out_dtype=None):
    """Forward projection of a device volume for plan views [a0, a1)."""
    a0, a1 = _range(plan, angle_range)
    _require(vol, plan.vol_shape, "volume")
    if vol.device.index != plan.device:
        raise ValueError("volume is on cuda:%s, plan on cuda:%d" % (vol.device.index, plan.device))
    proj_t = PROJECTORS.get(projection_type)
    if proj_t is None:
        raise ValueError("unknown projection_type %r" % (projection_type,))
    shape = (a1 - a0,) + plan.det_shape
    if out is None:
        out = torch.empty(shape, dtype=out_dtype or (vol.dtype if vol.dtype != torch.float16 else torch.float16),
                          device=vol.device)
    _require(out, shape, "projections")
    N.check(N.lib().tigre_ax(plan.handle, C.c_void_p(vol.data_ptr()), _dt(vol), C.c_void_p(out.data_ptr()),
                             _dt(out), proj_t, a0, a1, _stream(vol)), "tigre_ax")
    return out


def atb(proj: torch.Tensor, plan: "N.Plan", backprojection_type="FDK", angle_range=None, out=None, out_dtype=None):
    """Backprojection of device projections for plan views [a0, a1) (overwrites out)."""
    a0, a1 = _range(plan, angle_range)
    _require(proj, (a1 - a0,) + plan.det_shape, "projections")
    if proj.device.index != plan.device:
        raise ValueError("projections are on cuda:%s, plan on cuda:%d" % (proj.device.index, plan.device))
    bp = BACKPROJECTORS.get(backprojection_type)
    if bp is None:
        raise ValueError("unknown backprojection_type %r" % (backprojection_type,))
    if out is None:
        out = torch.empty(plan.vol_shape, dtype=out_dtype or proj.dtype, device=proj.device)
    _require(out, plan.vol_shape, "volume")
    N.check(N.lib().tigre_atb(plan.handle, C.c_void_p(proj.data_ptr()), _dt(proj), C.c_void_p(out.data_ptr()),
                              _dt(out), bp, a0, a1, _stream(proj)), "tigre_atb")
    return out


def siddon_segments(plan: "N.Plan", angle_range=None, device=None) -> int:
    """Total number of Siddon voxel segments over the plan's rays (FP64 setup only)."""
    a0, a1 = _range(plan, angle_range)
    dev = torch.device("cuda", plan.device)
    tot = torch.zeros(1, dtype=torch.int64, device=dev)
    N.check(N.lib().tigre_siddon_count_segments(plan.handle, a0, a1, C.c_void_p(tot.data_ptr()),
                                                C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)),
            "tigre_siddon_count_segments")
    return int(tot.item())


def interp_samples(plan: "N.Plan", angle_range=None) -> int:
    """Total number of interpolated samples inside the volume over the plan's rays (FP64 setup only)."""
    a0, a1 = _range(plan, angle_range)
    dev = torch.device("cuda", plan.device)
    tot = torch.zeros(1, dtype=torch.int64, device=dev)
    N.check(N.lib().tigre_interp_count_samples(plan.handle, a0, a1, C.c_void_p(tot.data_ptr()),
                                               C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)),
            "tigre_interp_count_samples")
    return int(tot.item())


def _vol3(t: torch.Tensor):
    if t.dim() != 3 or not t.is_cuda or not t.is_contiguous() or t.dtype != torch.float32:
        raise ValueError("expected a contiguous float32 CUDA volume (nZ, nY, nX)")
    nz, ny, nx = t.shape
    return nx, ny, nz


def tv_pocs_(vol: torch.Tensor, alpha: float, maxiter: int, work: torch.Tensor = None):
    """In-place POCS-TV descent (pocs_tv semantics) on a float32 device volume."""
    nx, ny, nz = _vol3(vol)
    if work is None:
        work = torch.empty_like(vol)
    N.check(N.lib().tigre_tv_pocs(C.c_void_p(vol.data_ptr()), N.F32, nx, ny, nz, float(alpha), int(maxiter),
                                  C.c_void_p(work.data_ptr()), _stream(vol)), "tigre_tv_pocs")
    return vol


def tv_aw_pocs_(vol: torch.Tensor, alpha: float, maxiter: int, delta: float, work: torch.Tensor = None):
    """In-place adaptive-weighted TV descent (aw_pocs_tv semantics) on a float32 device volume."""
    nx, ny, nz = _vol3(vol)
    if work is None:
        work = torch.empty_like(vol)
    N.check(N.lib().tigre_tv_aw_pocs(C.c_void_p(vol.data_ptr()), N.F32, nx, ny, nz, float(alpha), int(maxiter),
                                     float(delta), C.c_void_p(work.data_ptr()), _stream(vol)), "tigre_tv_aw_pocs")
    return vol


def tv_piccs_(vol: torch.Tensor, prior: torch.Tensor, alpha: float, ratio: float, maxiter: int,
              work: torch.Tensor = None):
    """In-place PICCS TV descent (piccs_tv semantics) on a float32 device volume with a device prior."""
    nx, ny, nz = _vol3(vol)
    if tuple(_vol3(prior)) != (nx, ny, nz):
        raise ValueError("prior and image sizes differ")
    if work is None:
        work = torch.empty_like(vol)
    N.check(N.lib().tigre_tv_piccs(C.c_void_p(vol.data_ptr()), C.c_void_p(prior.data_ptr()), N.F32, nx, ny, nz,
                                   float(alpha), float(ratio), int(maxiter), C.c_void_p(work.data_ptr()),
                                   _stream(vol)), "tigre_tv_piccs")
    return vol


def sart_update_(x: torch.Tensor, bp: torch.Tensor, v: torch.Tensor, lmbda: float, noneg: bool = True,
                 rounding: str = "nearest", seed: int = 0, step: int = 0):
    """In place x <- max(x + (lmbda / v) * bp, 0) on a device volume (tigre_sart_update).
    x: (nz, ny, nx) float32/bfloat16/float16; bp: float32 like x; v: float32 (ny, nx).
    rounding "stochastic" rounds 16-bit storage with Philox bits of (seed, step, voxel)."""
    if x.dim() != 3 or not x.is_cuda or not x.is_contiguous():
        raise ValueError("expected a contiguous CUDA volume (nZ, nY, nX)")
    nz, ny, nx = x.shape
    if bp.dtype != torch.float32 or tuple(bp.shape) != tuple(x.shape) or not bp.is_contiguous():
        raise ValueError("bp must be a contiguous float32 volume shaped like x")
    if v.dtype != torch.float32 or tuple(v.shape) != (ny, nx) or not v.is_contiguous():
        raise ValueError("v must be a contiguous float32 (ny, nx) plane")
    if bp.device != x.device or v.device != x.device:
        raise ValueError("x, bp and v must be on one device")
    mode = {"nearest": N.ROUND_NEAREST, "stochastic": N.ROUND_STOCHASTIC}[rounding]
    N.check(N.lib().tigre_sart_update(C.c_void_p(x.data_ptr()), _dt(x), C.c_void_p(bp.data_ptr()),
                                      C.c_void_p(v.data_ptr()), float(lmbda), 1 if noneg else 0, nz, ny * nx, mode,
                                      int(seed) & (2 ** 64 - 1), int(step) & (2 ** 64 - 1), _stream(x)),
            "tigre_sart_update")
    return x


def tv_gradient(vol: torch.Tensor, out: torch.Tensor = None):
    nx, ny, nz = _vol3(vol)
    if out is None:
        out = torch.empty_like(vol)
    N.check(N.lib().tigre_tv_gradient(C.c_void_p(vol.data_ptr()), N.F32, C.c_void_p(out.data_ptr()), nx, ny, nz,
                                      _stream(vol)), "tigre_tv_gradient")
    return out


def tv_value(vol: torch.Tensor) -> torch.Tensor:
    nx, ny, nz = _vol3(vol)
    out = torch.zeros((), dtype=torch.float64, device=vol.device)
    N.check(N.lib().tigre_tv_value(C.c_void_p(vol.data_ptr()), N.F32, nx, ny, nz, C.c_void_p(out.data_ptr()),
                                   _stream(vol)), "tigre_tv_value")
    return out


def sumsq(x: torch.Tensor, out: torch.Tensor = None) -> torch.Tensor:
    """FP64 sum of squares (accumulated into out when given)."""
    if out is None:
        out = torch.zeros((), dtype=torch.float64, device=x.device)
    N.check(N.lib().tigre_sumsq(C.c_void_p(x.data_ptr()), _dt(x), x.numel(), C.c_void_p(out.data_ptr()),
                                _stream(x)), "tigre_sumsq")
    return out


def dot(x: torch.Tensor, y: torch.Tensor, out: torch.Tensor = None) -> torch.Tensor:
    if x.dtype != torch.float32 or y.dtype != torch.float32 or x.numel() != y.numel():
        raise ValueError("dot takes two float32 tensors of equal size")
    if out is None:
        out = torch.zeros((), dtype=torch.float64, device=x.device)
    N.check(N.lib().tigre_dot(C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()), x.numel(),
                              C.c_void_p(out.data_ptr()), _stream(x)), "tigre_dot")
    return out
