"""ctypes binding of libtigre_b200.so (include/tigre_b200.h).

The library is built in-tree by tigre_b200._build; importing this module
loads it and fails loudly when it is missing -- there is no fallback path.
"""
from __future__ import annotations

import contextlib
import copy
import ctypes as C
import hashlib
import os
import threading

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libtigre_b200.so")

F32, BF16, F16 = 0, 1, 2
ROUND_NEAREST, ROUND_STOCHASTIC = 0, 1
PROJ_SIDDON, PROJ_INTERPOLATED = 0, 1
BACKPROJ_FDK, BACKPROJ_MATCHED = 0, 1
PLAN_PARALLEL = 1
STATUS_WAIT_EXPIRED, STATUS_RAY_DROPPED = 1, 2
# library options (tigre_set_option)
OPT_SIDDON_KERNEL, OPT_BP_BOX, OPT_BP_KERNEL, OPT_HOST_CHUNK_VIEWS, OPT_HOST_STAGING, OPT_BP_SKIP_COPY = 1, 2, 3, 4, 5, 6
OPT_INTERP_TEXTURE = 7

_FP = C.POINTER(C.c_float)


class TigreGeometry(C.Structure):
    """Field-for-field struct Geometry (Common/CUDA/types_TIGRE.hpp:48-85)."""

    _fields_ = [
        ("nVoxelX", C.c_int), ("nVoxelY", C.c_int), ("nVoxelZ", C.c_int),
        ("sVoxelX", C.c_float), ("sVoxelY", C.c_float), ("sVoxelZ", C.c_float),
        ("dVoxelX", C.c_float), ("dVoxelY", C.c_float), ("dVoxelZ", C.c_float),
        ("offOrigX", _FP), ("offOrigY", _FP), ("offOrigZ", _FP),
        ("DSO", _FP),
        ("nDetecU", C.c_int), ("nDetecV", C.c_int),
        ("sDetecU", C.c_float), ("sDetecV", C.c_float),
        ("dDetecU", C.c_float), ("dDetecV", C.c_float),
        ("offDetecU", _FP), ("offDetecV", _FP),
        ("DSD", _FP),
        ("dRoll", _FP), ("dPitch", _FP), ("dYaw", _FP),
        ("unitX", C.c_float), ("unitY", C.c_float), ("unitZ", C.c_float),
        ("alpha", C.c_float), ("theta", C.c_float), ("psi", C.c_float),
        ("COR", _FP),
        ("maxLength", C.c_float),
        ("accuracy", C.c_float),
    ]


class NativeError(RuntimeError):
    def __init__(self, code, where, msg):
        super().__init__("%s failed with code %d: %s" % (where, code, msg))
        self.code = code


_lib = None
_lock = threading.Lock()

_SIGS = {
    "tigre_last_error": (C.c_char_p, []),
    "tigre_version": (C.c_int, []),
    "tigre_launch_count": (C.c_ulonglong, []),
    "tigre_siddon_ray_projection": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p,
                                              C.c_int]),
    "tigre_interpolation_projection": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                                 C.c_void_p, C.c_int]),
    "tigre_voxel_backprojection": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p,
                                             C.c_int]),
    "tigre_voxel_backprojection2": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p,
                                              C.c_int]),
    "tigre_pocs_tv": (C.c_int, [C.c_void_p, C.c_void_p, C.c_float, C.c_void_p, C.c_int, C.c_void_p, C.c_int]),
    "tigre_siddon_ray_projection_parallel": (C.c_int, [C.c_void_p] * 4 + [C.c_int, C.c_void_p, C.c_int]),
    "tigre_interpolation_projection_parallel": (C.c_int, [C.c_void_p] * 4 + [C.c_int, C.c_void_p, C.c_int]),
    "tigre_voxel_backprojection_parallel": (C.c_int, [C.c_void_p] * 4 + [C.c_int, C.c_void_p, C.c_int]),
    "tigre_plan_create": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    "tigre_plan_create_ex": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    "tigre_plan_destroy": (None, [C.c_void_p]),
    "tigre_plan_scratch_bytes": (C.c_longlong, [C.c_void_p]),
    "tigre_plan_status": (C.c_int, [C.c_void_p, C.c_int]),
    "tigre_ax": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int,
                           C.c_void_p]),
    "tigre_atb": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int,
                            C.c_void_p]),
    "tigre_atb_ex": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int,
                               C.c_int, C.c_void_p]),
    "tigre_release_cache": (None, []),
    "tigre_set_option": (C.c_longlong, [C.c_int, C.c_longlong]),
    "tigre_get_option": (C.c_longlong, [C.c_int]),
    "tigre_siddon_count_segments": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p]),
    "tigre_interp_count_samples": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p]),
    "tigre_tv_pocs": (C.c_int, [C.c_void_p, C.c_int, C.c_long, C.c_long, C.c_long, C.c_float, C.c_int, C.c_void_p,
                                C.c_void_p]),
    "tigre_tv_pocs_noalloc": (C.c_int, [C.c_void_p, C.c_int, C.c_long, C.c_long, C.c_long, C.c_float, C.c_int,
                                        C.c_void_p, C.c_void_p]),
    "tigre_tvdenoising": (C.c_int, [C.c_void_p, C.c_void_p, C.c_float, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p,
                                    C.c_int]),
    "tigre_aw_pocs_tv": (C.c_int, [C.c_void_p, C.c_void_p, C.c_float, C.c_void_p, C.c_int, C.c_float, C.c_void_p,
                                   C.c_int]),
    "tigre_piccs_tv": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_float, C.c_float, C.c_void_p, C.c_int,
                                 C.c_void_p, C.c_int]),
    "tigre_tv_aw_pocs": (C.c_int, [C.c_void_p, C.c_int, C.c_long, C.c_long, C.c_long, C.c_float, C.c_int, C.c_float,
                                   C.c_void_p, C.c_void_p]),
    "tigre_tv_piccs": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_long, C.c_long, C.c_long, C.c_float, C.c_float,
                                 C.c_int, C.c_void_p, C.c_void_p]),
    "tigre_sart_update": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_float, C.c_int, C.c_longlong,
                                    C.c_longlong, C.c_int, C.c_ulonglong, C.c_ulonglong, C.c_void_p]),
    "tigre_noise_1d": (C.c_int, [C.c_void_p, C.c_longlong, C.c_int, C.c_float, C.c_float, C.c_ulonglong, C.c_void_p,
                                 C.c_void_p, C.c_int]),
    "tigre_add_noise": (C.c_int, [C.c_void_p, C.c_void_p, C.c_longlong, C.c_int, C.c_float, C.c_float,
                                  C.c_ulonglong, C.c_void_p]),
    "tigre_philox4x32": (C.c_int, [C.c_void_p, C.c_longlong, C.c_ulonglong, C.c_ulonglong, C.c_void_p]),
    "tigre_conv3d_col_elems": (C.c_longlong, [C.c_long, C.c_long, C.c_long, C.c_long]),
    "tigre_conv3d_set_tcgen05": (C.c_int, [C.c_int]),
    "tigre_conv3d_status": (C.c_int, [C.c_int]),
    "tigre_unet_pool2": (C.c_int, [C.c_void_p, C.c_void_p, C.c_long, C.c_long, C.c_long, C.c_long, C.c_void_p]),
    "tigre_unet_up_concat": (C.c_int, [C.c_void_p, C.c_long, C.c_void_p, C.c_long, C.c_void_p, C.c_long, C.c_long,
                                       C.c_long, C.c_void_p]),
    "tigre_unet_conv_in": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_long, C.c_long, C.c_long,
                                     C.c_long, C.c_int, C.c_void_p]),
    "tigre_unet_conv_out": (C.c_int, [C.c_void_p, C.c_long, C.c_void_p, C.c_float, C.c_void_p, C.c_void_p, C.c_long,
                                      C.c_long, C.c_long, C.c_void_p]),
    "tigre_conv3d_fwd": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_long, C.c_long,
                                   C.c_long, C.c_long, C.c_long, C.c_int, C.c_void_p, C.c_void_p]),
    "tigre_conv3d_bwd_data": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_long, C.c_long, C.c_long, C.c_long,
                                        C.c_long, C.c_void_p, C.c_void_p]),
    "tigre_conv3d_bwd_weight": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_long, C.c_long, C.c_long, C.c_long,
                                          C.c_long, C.c_void_p, C.c_void_p]),
    "tigre_tv_denoise_work_floats": (C.c_longlong, [C.c_long, C.c_long, C.c_long]),
    "tigre_tv_denoise": (C.c_int, [C.c_void_p, C.c_void_p, C.c_long, C.c_long, C.c_long, C.c_float, C.c_void_p,
                                   C.c_int, C.c_void_p, C.c_void_p]),
    "tigre_tv_gradient": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_long, C.c_long, C.c_long, C.c_void_p]),
    "tigre_tv_value": (C.c_int, [C.c_void_p, C.c_int, C.c_long, C.c_long, C.c_long, C.c_void_p, C.c_void_p]),
    "tigre_sumsq": (C.c_int, [C.c_void_p, C.c_int, C.c_long, C.c_void_p, C.c_void_p]),
    "tigre_dot": (C.c_int, [C.c_void_p, C.c_void_p, C.c_long, C.c_void_p, C.c_void_p]),
    "tigre_cgls_step": (C.c_int, [C.c_void_p, C.c_void_p, C.c_long, C.c_void_p, C.c_void_p, C.c_long, C.c_void_p,
                                  C.c_void_p, C.c_void_p, C.c_void_p]),
    "tigre_cgls_direction": (C.c_int, [C.c_void_p, C.c_void_p, C.c_long, C.c_void_p, C.c_void_p, C.c_void_p]),
    "tigre_convert": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_long, C.c_void_p]),
}


def lib():
    """Load libtigre_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        with _lock:
            if _lib is None:
                if not os.path.exists(LIB_PATH):
                    raise ImportError(
                        "libtigre_b200.so is not built (expected at %s); run `python -m tigre_b200._build`" % LIB_PATH)
                L = C.CDLL(LIB_PATH)
                for name, (res, args) in _SIGS.items():
                    fn = getattr(L, name)
                    fn.restype = res
                    fn.argtypes = args
                _lib = L
    return _lib


def exported_symbols():
    return list(_SIGS)


def last_error() -> str:
    return lib().tigre_last_error().decode(errors="replace")


def check(rc, where):
    if rc != 0:
        raise NativeError(rc, where, last_error())


# ------------------------------------------------------------------ geometry --
class CGeometry:
    """C geometry built from a checked Python geometry, following
    Python/tigre/utilities/cuda_interface/_types.pxd:69-166 (axis swap,
    per-angle arrays).  Keeps the float32 arrays alive."""

    def __init__(self, geo, n):
        self._keep = []

        def arr(v):
            a = np.ascontiguousarray(np.asarray(v, dtype=np.float32).reshape(n))
            self._keep.append(a)
            return a.ctypes.data_as(_FP)

        off = np.asarray(geo.offOrigin, dtype=np.float32).reshape(n, 3)
        offd = np.asarray(geo.offDetector, dtype=np.float32).reshape(n, 2)
        rot = np.asarray(geo.rotDetector, dtype=np.float32).reshape(n, 3)
        s = TigreGeometry()
        s.nVoxelX, s.nVoxelY, s.nVoxelZ = int(geo.nVoxel[2]), int(geo.nVoxel[1]), int(geo.nVoxel[0])
        s.sVoxelX, s.sVoxelY, s.sVoxelZ = float(geo.sVoxel[2]), float(geo.sVoxel[1]), float(geo.sVoxel[0])
        s.dVoxelX, s.dVoxelY, s.dVoxelZ = float(geo.dVoxel[2]), float(geo.dVoxel[1]), float(geo.dVoxel[0])
        s.offOrigX, s.offOrigY, s.offOrigZ = arr(off[:, 2]), arr(off[:, 1]), arr(off[:, 0])
        s.DSO = arr(geo.DSO)
        s.nDetecU, s.nDetecV = int(geo.nDetector[1]), int(geo.nDetector[0])
        s.sDetecU, s.sDetecV = float(geo.sDetector[1]), float(geo.sDetector[0])
        s.dDetecU, s.dDetecV = float(geo.dDetector[1]), float(geo.dDetector[0])
        s.offDetecU, s.offDetecV = arr(offd[:, 1]), arr(offd[:, 0])
        s.DSD = arr(geo.DSD)
        s.dRoll, s.dPitch, s.dYaw = arr(rot[:, 2]), arr(rot[:, 1]), arr(rot[:, 0])
        s.unitX = s.unitY = s.unitZ = 1.0
        s.COR = arr(geo.COR)
        s.accuracy = float(geo.accuracy)
        self.s = s


def checked_geometry(geo, angles):
    """deepcopy + check_geo + cast_to_single, as tigre.Ax/Atb do (Ax.py:43-50)."""
    g = copy.deepcopy(geo)
    g.check_geo(angles)
    g.cast_to_single()
    return g


def _geo_key(g, device):
    h = hashlib.sha1()
    for name in ("nVoxel", "sVoxel", "dVoxel", "nDetector", "sDetector", "dDetector", "DSO", "DSD", "offOrigin",
                 "offDetector", "rotDetector", "COR", "angles"):
        a = np.ascontiguousarray(np.asarray(getattr(g, name)))
        h.update(name.encode())
        h.update(str(a.dtype).encode() + str(a.shape).encode())
        h.update(a.tobytes())
    h.update(str(float(g.accuracy)).encode())
    h.update(str(getattr(g, "mode", "cone")).encode())
    h.update(str(device).encode())
    return h.hexdigest()


class Plan:
    """Owner of a TigrePlan: FP64 per-angle frames on one device + scratch."""

    def __init__(self, geo_checked, device=0):
        self.geo = geo_checked
        self.angles = np.ascontiguousarray(np.asarray(geo_checked.angles, dtype=np.float32).reshape(-1, 3))
        self.n = self.angles.shape[0]
        self.device = int(device)
        self._cg = CGeometry(geo_checked, self.n)
        h = C.c_void_p()
        self.parallel = getattr(geo_checked, "mode", "cone") == "parallel"
        check(lib().tigre_plan_create_ex(C.byref(self._cg.s), self.angles.ctypes.data, self.n, self.device,
                                         PLAN_PARALLEL if self.parallel else 0, C.byref(h)), "tigre_plan_create_ex")
        self.handle = h
        self.vol_shape = tuple(int(v) for v in geo_checked.nVoxel)
        self.det_shape = tuple(int(v) for v in geo_checked.nDetector)

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and _lib is not None:
            try:
                _lib.tigre_plan_destroy(h)
            except Exception:
                pass
            self.handle = None

    def scratch_bytes(self):
        return int(lib().tigre_plan_scratch_bytes(self.handle))

    def status(self, reset=True):
        """Kernel status word (0 = ok); synchronises the device."""
        return int(lib().tigre_plan_status(self.handle, 1 if reset else 0))


_plan_cache: "dict[str, Plan]" = {}
_PLAN_CACHE_MAX = 16


def get_plan(geo_checked, device=0) -> Plan:
    key = _geo_key(geo_checked, device)
    p = _plan_cache.get(key)
    if p is None:
        if len(_plan_cache) >= _PLAN_CACHE_MAX:
            _plan_cache.pop(next(iter(_plan_cache)))
        p = Plan(geo_checked, device)
        _plan_cache[key] = p
    return p


def clear_plan_cache():
    _plan_cache.clear()


def release_all():
    """Drops this module's plans and the host entry points' cached plans and buffers."""
    clear_plan_cache()
    lib().tigre_release_cache()


@contextlib.contextmanager
def option(key, value):
    """Sets a library option (TIGRE_OPT_*) for the duration of a block.  Plans read some
    options when they are created, so cached plans are dropped on entry and on exit."""
    L = lib()
    old = L.tigre_set_option(int(key), int(value))
    if old == -1 and L.tigre_get_option(int(key)) != int(value):
        raise ValueError("unknown option %d: %s" % (key, last_error()))
    release_all()
    try:
        yield
    finally:
        L.tigre_set_option(int(key), int(old))
        release_all()


def host_empty(shape):
    """float32 numpy array for a host-path result, in page-locked memory when a
    GPU is present (device->host copies into pageable memory go through a
    driver bounce buffer at a fraction of the link rate).  The pages come from
    torch's caching host allocator, so repeated calls of one size reuse them;
    the array keeps its tensor alive."""
    try:
        import torch
        if torch.cuda.is_available():
            return torch.empty(tuple(shape), dtype=torch.float32, pin_memory=True).numpy()
    except ImportError:
        pass
    return np.empty(tuple(shape), dtype=np.float32)
