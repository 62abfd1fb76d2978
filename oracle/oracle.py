"""ctypes front end of the FP64 host oracle (oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg, never by the product package.

Geometry conversion follows Python/tigre/utilities/cuda_interface/_types.pxd:69-166
(axis swap (z,y,x) -> x/y/z, (v,u) -> u/v; rotDetector[:,2]/[1]/[0] -> roll/pitch/yaw)
after the reference's check_geo() + cast_to_single().
"""
from __future__ import annotations

import copy
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

_D = C.POINTER(C.c_double)


class OGeo(C.Structure):
    _fields_ = [
        ("nVoxelX", C.c_int), ("nVoxelY", C.c_int), ("nVoxelZ", C.c_int),
        ("sVoxelX", C.c_double), ("sVoxelY", C.c_double), ("sVoxelZ", C.c_double),
        ("dVoxelX", C.c_double), ("dVoxelY", C.c_double), ("dVoxelZ", C.c_double),
        ("nDetecU", C.c_int), ("nDetecV", C.c_int),
        ("sDetecU", C.c_double), ("sDetecV", C.c_double),
        ("dDetecU", C.c_double), ("dDetecV", C.c_double),
        ("accuracy", C.c_double),
        ("nangles", C.c_int),
        ("offOrigX", _D), ("offOrigY", _D), ("offOrigZ", _D),
        ("offDetecU", _D), ("offDetecV", _D),
        ("DSO", _D), ("DSD", _D),
        ("dRoll", _D), ("dPitch", _D), ("dYaw", _D),
        ("COR", _D),
        ("alpha", _D), ("theta", _D), ("psi", _D),
    ]


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "_build", "liboracle.so")
        if not os.path.exists(path):
            import importlib.util
            spec = importlib.util.spec_from_file_location("_oracle_build", os.path.join(_HERE, "build.py"))
            mod = importlib.util.module_from_spec(spec)
            spec.loader.exec_module(mod)
            mod.build_oracle()
        _LIB = C.CDLL(path)
        f = C.c_void_p
        _LIB.oracle_siddon.argtypes = [f, C.POINTER(OGeo), C.c_int, C.c_int, C.c_int, C.c_int, f, f, C.c_int]
        _LIB.oracle_interp.argtypes = [f, C.POINTER(OGeo), C.c_int, C.c_int, C.c_int, C.c_int, f, f, C.c_int]
        _LIB.oracle_backproject.argtypes = [f, C.POINTER(OGeo), C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, f,
                                            C.c_int]
        _LIB.oracle_siddon_parallel.argtypes = [f, C.POINTER(OGeo), C.c_int, C.c_int, C.c_int, C.c_int, f, C.c_int]
        _LIB.oracle_interp_parallel.argtypes = [f, C.POINTER(OGeo), C.c_int, C.c_int, C.c_int, C.c_int, f, C.c_int]
        _LIB.oracle_backproject_parallel.argtypes = [f, C.POINTER(OGeo), C.c_int, C.c_int, C.c_int, C.c_int, f,
                                                     C.c_int]
        _LIB.oracle_tv_gradient.argtypes = [f, C.c_long, C.c_long, C.c_long, f, C.c_int]
        _LIB.oracle_pocs_tv.argtypes = [f, f, C.c_float, C.c_long, C.c_long, C.c_long, C.c_int, C.c_int]
        _LIB.oracle_aw_pocs_tv.argtypes = [f, f, C.c_float, C.c_float, C.c_long, C.c_long, C.c_long, C.c_int,
                                           C.c_int]
        _LIB.oracle_piccs_tv.argtypes = [f, f, f, C.c_float, C.c_float, C.c_long, C.c_long, C.c_long, C.c_int,
                                         C.c_int]
    return _LIB


class _Geo:
    """Keeps the per-angle double arrays alive while the C struct points at them."""

    def __init__(self, geo, angles):
        g = copy.deepcopy(geo)
        g.check_geo(angles)
        g.cast_to_single()
        n = g.angles.shape[0]
        self.n = n
        keep = {}

        def arr(v):
            a = np.ascontiguousarray(np.asarray(v, dtype=np.float64).reshape(n))
            keep[id(a)] = a
            return a.ctypes.data_as(_D)

        off = np.asarray(g.offOrigin, dtype=np.float64).reshape(n, 3)
        offd = np.asarray(g.offDetector, dtype=np.float64).reshape(n, 2)
        rot = np.asarray(g.rotDetector, dtype=np.float64).reshape(n, 3)
        ang = np.asarray(g.angles, dtype=np.float32).astype(np.float64).reshape(n, 3)
        s = OGeo()
        s.nVoxelX, s.nVoxelY, s.nVoxelZ = int(g.nVoxel[2]), int(g.nVoxel[1]), int(g.nVoxel[0])
        s.sVoxelX, s.sVoxelY, s.sVoxelZ = float(g.sVoxel[2]), float(g.sVoxel[1]), float(g.sVoxel[0])
        s.dVoxelX, s.dVoxelY, s.dVoxelZ = float(g.dVoxel[2]), float(g.dVoxel[1]), float(g.dVoxel[0])
        s.nDetecU, s.nDetecV = int(g.nDetector[1]), int(g.nDetector[0])
        s.sDetecU, s.sDetecV = float(g.sDetector[1]), float(g.sDetector[0])
        s.dDetecU, s.dDetecV = float(g.dDetector[1]), float(g.dDetector[0])
        s.accuracy = float(g.accuracy)
        s.nangles = n
        s.offOrigX, s.offOrigY, s.offOrigZ = arr(off[:, 2]), arr(off[:, 1]), arr(off[:, 0])
        s.offDetecU, s.offDetecV = arr(offd[:, 1]), arr(offd[:, 0])
        s.DSO, s.DSD = arr(g.DSO), arr(g.DSD)
        s.dRoll, s.dPitch, s.dYaw = arr(rot[:, 2]), arr(rot[:, 1]), arr(rot[:, 0])
        s.COR = arr(g.COR)
        s.alpha, s.theta, s.psi = arr(ang[:, 0]), arr(ang[:, 1]), arr(ang[:, 2])
        self.s = s
        self._keep = keep
        self.g = g


def _threads(nthreads):
    return int(nthreads) if nthreads else (os.cpu_count() or 1)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def ax(img, geo, angles, projection_type="Siddon", angle_range=None, row_range=None, nthreads=0,
       return_counts=False):
    """FP64 forward projection.  Returns (nA, nR, nU) float32 for the selected angles/rows
    (and the per-ray segment/sample counts when return_counts)."""
    G = _Geo(geo, angles)
    s = G.s
    a0, a1 = angle_range if angle_range is not None else (0, G.n)
    v0, v1 = row_range if row_range is not None else (0, s.nDetecV)
    img = _f32(img)
    assert img.shape == (s.nVoxelZ, s.nVoxelY, s.nVoxelX)
    out = np.zeros((a1 - a0, v1 - v0, s.nDetecU), dtype=np.float32)
    siddon = projection_type in ("Siddon", "ray-voxel")
    if getattr(G.g, "mode", "cone") == "parallel":
        assert not return_counts, "counts are kept for cone beam only"
        fn = lib().oracle_siddon_parallel if siddon else lib().oracle_interp_parallel
        fn(img.ctypes.data, C.byref(s), a0, a1, v0, v1, out.ctypes.data, _threads(nthreads))
        return out
    cnt = np.zeros(out.shape, dtype=np.int32) if return_counts else None
    fn = lib().oracle_siddon if siddon else lib().oracle_interp
    fn(img.ctypes.data, C.byref(s), a0, a1, v0, v1, out.ctypes.data,
       cnt.ctypes.data if cnt is not None else None, _threads(nthreads))
    return (out, cnt) if return_counts else out


def atb(proj, geo, angles, backprojection_type="FDK", angle_range=None, z_range=None, nthreads=0):
    """FP64 voxel backprojection of proj (nA, nV, nU).  Returns (nz, nY, nX) float32."""
    G = _Geo(geo, angles)
    s = G.s
    a0, a1 = angle_range if angle_range is not None else (0, G.n)
    z0, z1 = z_range if z_range is not None else (0, s.nVoxelZ)
    proj = _f32(proj)
    assert proj.shape == (G.n, s.nDetecV, s.nDetecU)
    out = np.zeros((z1 - z0, s.nVoxelY, s.nVoxelX), dtype=np.float32)
    if getattr(G.g, "mode", "cone") == "parallel":   # one parallel backprojector for both types
        lib().oracle_backproject_parallel(proj.ctypes.data, C.byref(s), a0, a1, z0, z1, out.ctypes.data,
                                          _threads(nthreads))
        return out
    matched = 1 if backprojection_type == "matched" else 0
    lib().oracle_backproject(proj.ctypes.data, C.byref(s), a0, a1, z0, z1, matched, out.ctypes.data,
                             _threads(nthreads))
    return out


def tv_gradient(img, nthreads=0):
    img = _f32(img)
    nz, ny, nx = img.shape
    out = np.empty_like(img)
    lib().oracle_tv_gradient(img.ctypes.data, nx, ny, nz, out.ctypes.data, _threads(nthreads))
    return out


def pocs_tv(img, alpha, maxiter, nthreads=0):
    img = _f32(img)
    nz, ny, nx = img.shape
    out = np.empty_like(img)
    lib().oracle_pocs_tv(img.ctypes.data, out.ctypes.data, float(alpha), nx, ny, nz, int(maxiter),
                         _threads(nthreads))
    return out


def aw_pocs_tv(img, alpha, maxiter, delta, nthreads=0):
    """aw_pocs_tv (Common/CUDA/GD_AwTV.cu:276-720) in FP64."""
    img = _f32(img)
    nz, ny, nx = img.shape
    out = np.empty_like(img)
    lib().oracle_aw_pocs_tv(img.ctypes.data, out.ctypes.data, float(alpha), float(delta), nx, ny, nz, int(maxiter),
                            _threads(nthreads))
    return out


def piccs_tv(img, prior, alpha, ratio, maxiter, nthreads=0):
    """piccs_tv (Common/CUDA/PICCS.cu:274-380) in FP64."""
    img, prior = _f32(img), _f32(prior)
    if prior.shape != img.shape:
        raise ValueError("prior and image sizes differ")
    nz, ny, nx = img.shape
    out = np.empty_like(img)
    lib().oracle_piccs_tv(img.ctypes.data, prior.ctypes.data, out.ctypes.data, float(alpha), float(ratio), nx, ny, nz,
                          int(maxiter), _threads(nthreads))
    return out


# ---------------------------------------------------------------- FDK pieces --
def fdk_filter(proj, geo, angles, filter=None, cosine=True, filter_scale=None,  # noqa: A002
               stop_before_filter=False):
    """Cosine weighting + ramp filtering exactly as the reference's host path:
    single_pass_algorithms.py:186-197 then filtering.py:15-53 (scipy.fft on
    complex64, two projections per transform).  cosine=False: the ramp filter
    alone, as fbp uses it (single_pass_algorithms.py:221).  filter_scale replaces
    the angular factor 2 pi / nangles; stop_before_filter returns the cosine-weighted
    projections."""
    from scipy.fft import fft, ifft
    g = copy.deepcopy(geo)
    g.check_geo(angles)
    nv, nu = int(g.nDetector[0]), int(g.nDetector[1])
    du, dv = float(g.dDetector[1]), float(g.dDetector[0])
    xv = np.arange(-nu / 2 + 0.5, 1 + nu / 2 - 0.5) * du
    yv = np.arange(-nv / 2 + 0.5, 1 + nv / 2 - 0.5) * dv
    yy, xx = np.meshgrid(xv, yv)
    dsd, dso = float(g.DSD[0]), float(g.DSO[0])
    w = dsd / np.sqrt(dsd ** 2 + xx ** 2 + yy ** 2) if cosine else np.ones_like(xx)
    p = np.multiply(np.asarray(proj, dtype=np.float32), w).astype(np.float32)
    if stop_before_filter:
        return p

    def nextpow2(n):
        i = 1
        while (2 ** i) <= n:
            i += 1
        return i

    L = max(64, 2 ** nextpow2(2 * nu))
    nn = np.arange(-L / 2, L / 2)
    h = np.zeros(nn.shape, dtype=np.float32)
    h[int(L / 2)] = 1 / 4
    odd = nn % 2 == 1
    h[odd] = -1 / (np.pi * nn[odd]) ** 2
    fk = abs(np.fft.fft(h)) * 2
    filt = fk[: int(L / 2 + 1)]
    wv = 2 * np.pi * np.arange(len(filt)) / L
    if filter == "shepp_logan":
        filt[1:] *= np.sin(wv[1:] / 2) / (wv[1:] / 2)
    elif filter == "cosine":
        filt[1:] *= np.cos(wv[1:] / 2)
    elif filter == "hamming":
        filt[1:] *= 0.54 + 0.46 * np.cos(wv[1:])
    elif filter == "hann":
        filt[1:] *= (1 + np.cos(wv[1:])) / 2
    filt[wv > np.pi] = 0
    filt = np.hstack((filt, filt[1:-1][::-1])).astype(np.float32)
    filt = np.kron(np.ones((nv, 1), dtype=np.float32), filt)
    pad = int((L - nu) // 2)
    n = p.shape[0]
    scale = (dsd / dso) * ((2 * np.pi / n) if filter_scale is None else filter_scale) / (4 * du)
    f = np.empty((nv, L), dtype=np.complex64)
    for i in range(0, n - 1, 2):
        f.fill(0)
        f.real[:, pad:pad + nu] = p[i]
        f.imag[:, pad:pad + nu] = p[i + 1]
        f = ifft(fft(f, axis=1) * filt, axis=1)
        p[i] = f.real[:, pad:pad + nu] * scale
        p[i + 1] = f.imag[:, pad:pad + nu] * scale
    if n % 2:
        f.fill(0)
        f.real[:, pad:pad + nu] = p[n - 1]
        f = np.real(ifft(fft(f, axis=1) * filt, axis=1))
        p[n - 1] = f[:, pad:pad + nu] * scale
    return p


def parker_weights(geo, angles, q=1.0):
    """FP64 Parker short-scan weights, (nangles, nU): Wesarg, Ebert and Bortfeld, "Parker
    weights revisited", Med. Phys. 29(3) 2002, as TIGRE restates them in
    MATLAB/Utilities/ParkerWeight.m:17-43 -- fan angle of each detector column along u,
    negated when the angles increase, half fan angle delta from the outermost column
    centres, overscan epsilon = max(span - (pi + 2 delta), 0), and the smooth step S of
    the four transition terms.  Python/tigre/utilities/parkerweight.py:23-78 evaluates
    the same expression (it always negates, and takes the extent of the first detector
    axis, so it agrees for square detectors with increasing angles: pinned against it by
    tests/golden/ref_parker.npz).  Divisions by a zero transition width follow IEEE
    arithmetic and S maps NaN to 0, as the reference's boolean masks do."""
    g = copy.deepcopy(geo)
    g.check_geo(angles)
    a = np.asarray(g.angles, dtype=np.float64)[:, 0]
    nu, du, su = int(g.nDetector[1]), float(g.dDetector[1]), float(g.sDetector[1])
    gam = np.arctan((np.arange(nu, dtype=np.float64) * du - su / 2 + du / 2) / float(np.mean(g.DSD)))
    if np.all(np.diff(a) >= 0):
        gam = -gam
    delta = abs(gam[-1] - gam[0]) / 2
    eps = max(abs(a[-1] - a[0]) - (np.pi + 2 * delta), 0.0)
    beta = np.abs(a - a[0])[:, None]

    def smooth_step(t):
        inner = 0.5 * (1.0 + np.sin(np.pi * np.clip(t, -0.5, 0.5)))
        return np.where(t >= 0.5, 1.0, np.where(np.abs(t) < 0.5, inner, 0.0))

    with np.errstate(divide="ignore", invalid="ignore"):
        wa = q * (2 * delta - 2 * gam + eps)
        wb = q * (2 * delta + 2 * gam + eps)
        w = 0.5 * (smooth_step(beta / wa - 0.5) + smooth_step((beta - 2 * delta + 2 * gam - eps) / wa + 0.5)
                   - smooth_step((beta - np.pi + 2 * gam) / wb - 0.5)
                   - smooth_step((beta - np.pi - 2 * delta - eps) / wb + 0.5))
    return w


def fdk(proj, geo, angles, filter=None, parker=False, z_range=None):  # noqa: A002
    """FDK: cosine weights, optional Parker weights (parker = q, True meaning 1), ramp
    filter, FDK-weighted backprojection.  With Parker weights the angular factor of the
    filter scale is 2 * mean view step instead of 2 pi / nangles
    (MATLAB/Utilities/filtering.m:23-26,47-48, the wiring of MATLAB/Algorithms/FDK.m:153-161)."""
    if not parker:
        return atb(fdk_filter(proj, geo, angles, filter), geo, angles, "FDK", z_range=z_range)
    q = 1.0 if parker is True else float(parker)
    a = np.asarray(angles, dtype=np.float64)
    a = a[:, 0] if a.ndim == 2 else a
    # fdk_filter applies cosine weights, then filters; Parker weights go between the two
    W = parker_weights(geo, angles, q)
    cos_only = fdk_filter(proj, geo, angles, filter, cosine=True, filter_scale=None, stop_before_filter=True)
    weighted = (cos_only.astype(np.float64) * W[:, None, :]).astype(np.float32)
    filt = fdk_filter(weighted, geo, angles, filter, cosine=False,
                      filter_scale=2 * float(np.mean(np.abs(np.diff(a)))))
    return atb(filt, geo, angles, "FDK", z_range=z_range)


def fbp(proj, geo, angles, filter=None):  # noqa: A002
    """Parallel-beam FBP of single_pass_algorithms.py:206-228: ramp filter, parallel
    backprojection, times DSO/DSD."""
    g = copy.deepcopy(geo)
    g.check_geo(angles)
    w = float(np.asarray(g.DSO).reshape(-1)[0]) / float(np.asarray(g.DSD).reshape(-1)[0])
    return (atb(fdk_filter(proj, geo, angles, filter, cosine=False), geo, angles, "FDK") * np.float32(w))


def tvdenoise(img, niter, lmbda, spacing=(1.0, 1.0, 1.0)):
    """TV denoising of tvdenoising (tv_proximal.cu:185-630, one device) in FP64: the image
    between a lower slice holding image slice 1 and an upper zero slice (cpy_from_host,
    :672-692), u = f, p = 0, then maxIter steps of update_u (:136-153) and update_p
    (:156-181) with the reference's FP32 step sizes.  spacing = (dX, dY, dZ)."""
    img = np.asarray(img, dtype=np.float64)
    nz = img.shape[0]
    dxs, dys, dzs = (float(v) for v in spacing)
    f = np.zeros((nz + 2,) + img.shape[1:], dtype=np.float64)
    if nz > 1:
        f[0] = img[1]
    f[1:nz + 1] = img
    u = f.copy()
    pz, py, px = np.zeros_like(u), np.zeros_like(u), np.zeros_like(u)
    for i in range(int(niter)):
        tau2 = np.float32(0.3) + np.float32(0.02) * np.float32(i)
        tau1 = (np.float32(1) / tau2) * (np.float32(1) / np.float32(6) - np.float32(5) / (np.float32(15) + np.float32(i)))
        tau1, tau2 = float(tau1), float(tau2)
        div = pz.copy()
        div[1:] = (pz[1:] - pz[:-1]) / dzs
        d = py.copy()
        d[:, 1:] = (py[:, 1:] - py[:, :-1]) / dys
        div += d
        d = px.copy()
        d[:, :, 1:] = (px[:, :, 1:] - px[:, :, :-1]) / dxs
        div += d
        u = u * (1.0 - tau1) + tau1 * (f + div / lmbda)
        gz = np.zeros_like(u); gz[:-1] = (u[1:] - u[:-1]) / dzs
        gy = np.zeros_like(u); gy[:, :-1] = (u[:, 1:] - u[:, :-1]) / dys
        gx = np.zeros_like(u); gx[:, :, :-1] = (u[:, :, 1:] - u[:, :, :-1]) / dxs
        qz, qy, qx = pz + tau2 * gz, py + tau2 * gy, px + tau2 * gx
        nrm = np.maximum(1.0, np.sqrt(qz * qz + qy * qy + qx * qx))
        pz, py, px = qz / nrm, qy / nrm, qx / nrm
    return u[1:nz + 1].astype(np.float32)


def im3ddenoise(img, niter=50, lmbda=15.0):
    """im_3d_denoise.py:7-27 over the oracle tvdenoise (min/max scaling)."""
    img = np.asarray(img, dtype=np.float32)
    lo = img.min()
    x = img - lo
    hi = x.max()
    x = x / hi
    return (tvdenoise(x, niter, lmbda) * hi + lo).astype(np.float32)


def fista(proj, geo, angles, niter, hyper, tviter=20, tvlambda=0.1):
    """FISTA of ista_algorithms.py:13-176 in FP64 over the oracle pair and oracle im3ddenoise."""
    b = np.asarray(proj, dtype=np.float64)
    x = np.zeros(tuple(int(v) for v in geo.nVoxel), dtype=np.float64)
    bm = 1.0 / hyper
    x_rec = x.copy()
    lam = 2.0 * bm * tvlambda
    t = 1.0
    for _ in range(niter):
        r = b - ax(x.astype(np.float32), geo, angles, "interpolated")
        x = np.maximum(x + 2.0 * bm * atb(r.astype(np.float32), geo, angles, "matched"), 0.0)
        x_old = x_rec
        x_rec = im3ddenoise(x.astype(np.float32), tviter, 1.0 / lam).astype(np.float64)
        t_old = t
        t = (1.0 + np.sqrt(1.0 + 4.0 * t * t)) / 2.0
        x = x_rec + (t_old - 1.0) / t * (x_rec - x_old)
    return x.astype(np.float32)


def mlem(proj, geo, angles, niter, x0=None):
    """MLEM of statistical_algorithms.py:11-55 in FP64 over the oracle pair (interpolated Ax,
    matched Atb)."""
    b = np.asarray(proj, dtype=np.float64)
    W = atb(np.ones(b.shape, dtype=np.float32), geo, angles, "matched").astype(np.float64)
    W[W <= 0.0] = np.inf
    shape = tuple(int(v) for v in geo.nVoxel)
    x = np.ones(shape, dtype=np.float64) if x0 is None else np.array(x0, dtype=np.float64)
    x[x < 0.0] = 0.0
    for _ in range(niter):
        den = ax(x.astype(np.float32), geo, angles, "interpolated").astype(np.float64)
        den[den == 0.0] = np.inf
        img = atb((b / den).astype(np.float32), geo, angles, "matched").astype(np.float64) / W
        x = x * img
        x[x < 0.0] = 0.0
    return x.astype(np.float32)


def ossart(proj, geo, angles, niter, index, lmbda=1.0, noneg=True, callback=None):
    """OS-SART with FP64 state over the oracle pair (Siddon Ax, FDK Atb):
    W of set_w (iterative_recon_alg.py:214-230), V of set_v (:232-270), the per-subset update of
    update_image (:372-401) and the clip of art_data_minimizing (:326-345).  index: the view
    subsets in update order (order_subsets).  callback(it, x) after every iteration (FP64 x)."""
    g = copy.deepcopy(geo)
    g.check_geo(angles)
    ang = np.asarray(g.angles, dtype=np.float64)
    b = np.asarray(proj, dtype=np.float64)
    parallel = getattr(g, "mode", "cone") == "parallel"

    def sub(idx):
        gs = copy.deepcopy(g)
        for name in ("offOrigin", "offDetector", "rotDetector", "DSD", "DSO", "COR"):
            setattr(gs, name, np.asarray(getattr(g, name))[idx])
        gs.angles = ang[idx]
        return gs

    gx = copy.deepcopy(g)
    sv = np.array(gx.sVoxel, dtype=np.float64)
    sv[1:] = sv[1:] * 1.1
    sv[0] = max(float(gx.sDetector[0]), sv[0])
    gx.sVoxel, gx.nVoxel = sv, np.array([2, 2, 2])
    gx.dVoxel = sv / gx.nVoxel
    W = ax(np.ones((2, 2, 2), dtype=np.float32), gx, ang, "Siddon").astype(np.float64)
    W[W <= min(np.asarray(g.dVoxel, dtype=np.float64) / 2)] = np.inf
    W = 1.0 / W
    nv, nu = int(g.nDetector[0]), int(g.nDetector[1])
    shape = tuple(int(v) for v in g.nVoxel)
    V = []
    for idx in index:
        idx = np.asarray(idx).reshape(-1)
        if parallel:
            v = np.full(shape[1:], float(len(idx)))
        else:
            gs = sub(idx)
            s2 = np.array(gs.sVoxel, dtype=np.float64)
            gs.sVoxel = s2 * np.max(s2[1:] / np.linalg.norm(s2[1:])) * 0.9
            gs.dVoxel = gs.sVoxel / gs.nVoxel
            v = atb(np.ones((len(idx), nv, nu), dtype=np.float32), gs, gs.angles, "FDK").astype(np.float64).mean(0)
        v[v == 0.0] = np.inf
        V.append(v)
    x = np.zeros(shape, dtype=np.float64)
    for it in range(niter):
        for j, idx in enumerate(index):
            idx = np.asarray(idx).reshape(-1)
            gs = sub(idx)
            est = ax(x.astype(np.float32), gs, gs.angles, "Siddon").astype(np.float64)
            err = W[idx] * (b[idx] - est)
            x = x + lmbda / V[j] * atb(err.astype(np.float32), gs, gs.angles, "FDK").astype(np.float64)
            if noneg:
                x[x < 0.0] = 0.0
        if callback is not None:
            callback(it, x)
    return x.astype(np.float32)


def _kry_ops(geo, angles):
    A = lambda v: ax(np.asarray(v, dtype=np.float32), geo, angles, "Siddon").astype(np.float64)  # noqa: E731
    At = lambda r: atb(np.asarray(r, dtype=np.float32), geo, angles, "matched").astype(np.float64)  # noqa: E731
    return A, At


def _kry_stop(i, l2, restart):
    return i > 0 and l2[i] > l2[i - 1] and (i == 1 or not restart)


def hybrid_lsqr(proj, geo, angles, niter, lmbda=1.0, restart=True):
    """hybrid_LSQR of krylov_subspace_algorithms.py:190-296 in FP64 (elementwise
    re-orthogonalisation kept); returns the last non-growing iterate."""
    A, At = _kry_ops(geo, angles)
    b = np.asarray(proj, dtype=np.float64)
    x = np.zeros(tuple(int(v) for v in geo.nVoxel))
    u = b - A(x)
    normr = np.linalg.norm(u)
    u = u / normr
    U, V = [u], []
    B = np.zeros((niter, niter + 1))
    rhs = np.zeros(niter + 1)
    rhs[0] = normr
    beta = normr
    l2, best = [], x
    for i in range(niter):
        v = At(u)
        if i > 0:
            v = v - beta * V[i - 1]
        for j in range(i - 1):
            v = v - V[j] * v * V[j]
        alpha = np.linalg.norm(v)
        v = v / alpha
        V.append(v)
        u = A(v) - alpha * u
        for j in range(i - 1):
            u = u - U[j] * u * U[j]
        beta = np.linalg.norm(u)
        u = u / beta
        U.append(u)
        B[i, i], B[i, i + 1] = alpha, beta
        Uk, Sk, Vh = np.linalg.svd(B[:i + 1, :i + 2].T)
        y = Vh.T @ (Sk * (Uk.T @ rhs[:i + 2])[:i + 1] / (Sk ** 2 + lmbda ** 2))
        xi = x + sum(V[j] * y[j] for j in range(i + 1))
        l2.append(np.linalg.norm(b - A(xi)))
        if _kry_stop(i, l2, restart):
            return best.astype(np.float32), np.asarray(l2[:-1])
        best = xi
    return best.astype(np.float32), np.asarray(l2)


def gmres(proj, geo, angles, niter, space, restart=True):
    """AB-GMRES (space='proj', :570-631) / BA-GMRES (space='vol', :634-695) with the matched
    backprojector, in FP64."""
    A, At = _kry_ops(geo, angles)
    b = np.asarray(proj, dtype=np.float64)
    x = np.zeros(tuple(int(v) for v in geo.nVoxel))
    r = b - A(x)
    if space == "vol":
        r = At(r)
    rn = np.linalg.norm(r)
    W = [r / rn]
    H = np.zeros((niter, niter + 1))
    l2, best = [], x
    for k in range(niter):
        q = A(At(W[k])) if space == "proj" else At(A(W[k]))
        for i in range(k + 1):
            H[k, i] = np.sum(q * W[i])
            q = q - H[k, i] * W[i]
        H[k, k + 1] = np.linalg.norm(q)
        W.append(q / H[k, k + 1])
        e1 = np.zeros(k + 2)
        e1[0] = rn
        y = np.linalg.lstsq(H[:k + 1, :k + 2].T, e1, rcond=None)[0]
        d = sum(W[i] * y[i] for i in range(k + 1))
        xi = x + (At(d) if space == "proj" else d)
        l2.append(np.linalg.norm(b - A(xi)))
        if _kry_stop(k, l2, restart):
            return best.astype(np.float32), np.asarray(l2[:-1])
        best = xi
    return best.astype(np.float32), np.asarray(l2)


def _irn_diffs(img):
    out = []
    for axis in range(3):
        d = img.copy()
        n = img.shape[axis]
        sl = [slice(None)] * 3
        lo, hi = list(sl), list(sl)
        lo[axis], hi[axis] = slice(0, n - 2), slice(1, n - 1)
        if n > 2:
            d[tuple(lo)] = img[tuple(lo)] - img[tuple(hi)]
        out.append(d)
    return out


def _irn_Lx(W, img):
    return np.stack([W * d for d in _irn_diffs(img)])


def _irn_Ltx(W, g3):
    acc = 0.0
    for axis in range(3):
        wg = W * g3[axis]
        o = wg.copy()
        n = wg.shape[axis]
        idx = lambda a, b_: tuple(slice(a, b_) if k == axis else slice(None) for k in range(3))  # noqa: E731
        if n > 3:
            o[idx(1, n - 2)] = wg[idx(1, n - 2)] - wg[idx(0, n - 3)]
        if n >= 2:
            o[idx(n - 1, n)] = -wg[idx(n - 2, n - 1)]
        acc = acc + o
    return acc


def irn_tv_cgls(proj, geo, angles, niter, lmbda=1.0, niter_outer=4):
    """IRN_TV_CGLS of krylov_subspace_algorithms.py:441-567 in FP64, with the reference's
    difference operators (:466-500) and its restart-from-res0 bookkeeping."""
    A, At = _kry_ops(geo, angles)
    b = np.asarray(proj, dtype=np.float64)
    sl = np.sqrt(lmbda)
    x = np.zeros(tuple(int(v) for v in geo.nVoxel))
    x0 = x
    l2 = []
    for _ in range(niter_outer):
        d = _irn_diffs(x)
        W = (d[0] ** 2 + d[1] ** 2 + d[2] ** 2 + 1e-6) ** (-0.25)
        x = x0
        r1 = b - A(x)
        r2 = -_irn_Lx(W, x) * sl
        p = At(r1) + sl * _irn_Ltx(W, r2)
        gamma = np.sum(p * p)
        for _i in range(niter):
            x0 = x
            q1 = A(p)
            q2 = _irn_Lx(W, p) * sl
            alpha = gamma / (np.sum(q1 * q1) + np.sum(q2 * q2))
            x = x + alpha * p
            l2.append(np.linalg.norm(b - A(x)))
            r1 = r1 - alpha * q1
            r2 = r2 - alpha * q2
            s_ = At(r1) + sl * _irn_Ltx(W, r2)
            gamma1 = np.sum(s_ * s_)
            p = s_ + gamma1 / gamma * p
            gamma = gamma1
    return x.astype(np.float32), np.asarray(l2)


def hybrid_flsqr_tv(proj, geo, angles, niter, lmbda=1.0, restart=True):
    """hybrid_fLSQR_TV of krylov_subspace_algorithms.py:698-858 in FP64, with the inner
    scipy.sparse.linalg.lsqr solves (iter_lim=50) the reference makes; returns the iterate (the
    reference computes it and its decorator discards it)."""
    from scipy.sparse.linalg import LinearOperator, lsqr as sp_lsqr
    A, At = _kry_ops(geo, angles)
    b = np.asarray(proj, dtype=np.float64)
    shape = tuple(int(v) for v in geo.nVoxel)
    N = int(np.prod(shape))
    x = np.zeros(shape)
    u = b - A(x)
    k_aux = A(np.ones(shape) / np.sqrt(N))
    kn2 = np.sum(k_aux * k_aux)
    xA0 = np.ones(shape) * (np.sum(k_aux * u) / (np.sqrt(N) * kn2))
    k_aux = At(k_aux) / (np.sqrt(N) * kn2)
    u = u - A(xA0)
    normr = np.linalg.norm(u)
    u = u / normr
    U, V, Z = [u], [], []
    M = np.zeros((niter, niter + 1))
    rhs = np.zeros(niter + 1)
    rhs[0] = normr
    W = np.ones(shape) if x.max() == 0 else None
    Lx = lambda t: _irn_Lx(W, t.reshape(shape)).ravel()  # noqa: E731
    Ltx = lambda t: _irn_Ltx(W, t.reshape((3,) + shape)).ravel()  # noqa: E731
    l2, best = [], x + xA0
    for i in range(niter):
        v = At(u)
        for j in range(i):
            v = v - np.sum(V[j] * v) * V[j]
        v = v / np.linalg.norm(v)
        zt = v.ravel() - k_aux.ravel() * np.sum(v)
        op1 = LinearOperator((N, 3 * N), matvec=Ltx, rmatvec=Lx, dtype=np.float64)
        aux = sp_lsqr(op1, zt, iter_lim=50)[0]
        op2 = LinearOperator((3 * N, N), matvec=Lx, rmatvec=Ltx, dtype=np.float64)
        zt = sp_lsqr(op2, aux, iter_lim=50)[0]
        zt = (zt - np.sum(k_aux.ravel() * zt)).reshape(shape)
        V.append(v)
        Z.append(zt)
        u = A(zt)
        for j in range(i + 1):
            M[i, j] = np.sum(U[j] * u)
            u = u - M[i, j] * U[j]
        M[i, i + 1] = np.linalg.norm(u)
        u = u / M[i, i + 1]
        U.append(u)
        WZ = np.stack([Lx(Z[j]) for j in range(i + 1)], axis=1)
        R = np.linalg.qr(WZ, mode="r")
        MZ = np.concatenate([M[:i + 1, :i + 2].T, lmbda * R])
        rz = np.concatenate([rhs[:i + 2], np.zeros(i + 1)])
        y = np.linalg.lstsq(MZ, rz, rcond=None)[0]
        xi = x + xA0 + sum(Z[j] * y[j] for j in range(i + 1))
        l2.append(np.linalg.norm(b - A(xi)))
        if _kry_stop(i, l2, restart):
            return best.astype(np.float32), np.asarray(l2[:-1])
        best = xi
    return best.astype(np.float32), np.asarray(l2)


def lsqr(proj, geo, angles, niter):
    """LSQR of krylov_subspace_algorithms.py:101-187 with FP64 vectors over the oracle pair."""
    A = lambda v: ax(v.astype(np.float32), geo, angles, "Siddon").astype(np.float64)  # noqa: E731
    At = lambda r: atb(r.astype(np.float32), geo, angles, "matched").astype(np.float64)  # noqa: E731
    b = np.asarray(proj, dtype=np.float64)
    x = np.zeros(tuple(int(v) for v in geo.nVoxel), dtype=np.float64)
    u = b.copy(); beta = np.linalg.norm(u); u /= beta; phibar = beta
    v = At(u); alpha = np.linalg.norm(v); v /= alpha; rhobar = alpha; w = v.copy()
    res = []
    for _ in range(niter):
        u = A(v) - alpha * u; beta = np.linalg.norm(u); u /= beta
        v = At(u) - beta * v; alpha = np.linalg.norm(v); v /= alpha
        rho = np.hypot(rhobar, beta); c, s = rhobar / rho, beta / rho
        theta = s * alpha; rhobar = -c * alpha; phi = c * phibar; phibar = s * phibar
        x += (phi / rho) * w; w_old = w; w = v - (theta / rho) * w
        rn = np.linalg.norm(b - A(x))
        if res and rn > res[-1]:
            x -= (phi / rho) * w_old
            break
        res.append(rn)
    return x.astype(np.float32), np.asarray(res)


def lsmr(proj, geo, angles, niter, lmbda=1.0):
    """LSMR of krylov_subspace_algorithms.py:299-439 with FP64 vectors over the oracle pair."""
    A = lambda v: ax(v.astype(np.float32), geo, angles, "Siddon").astype(np.float64)  # noqa: E731
    At = lambda r: atb(r.astype(np.float32), geo, angles, "matched").astype(np.float64)  # noqa: E731
    b = np.asarray(proj, dtype=np.float64)
    x = np.zeros(tuple(int(v) for v in geo.nVoxel), dtype=np.float64)
    u = b.copy(); beta = np.linalg.norm(u); u /= beta
    v = At(u); alpha = np.linalg.norm(v); v /= alpha
    alphabar, zetabar, rho, rhobar, cbar, sbar = alpha, alpha * beta, 1.0, 1.0, 1.0, 0.0
    h = v.copy(); hbar = np.zeros_like(h)
    res = []
    for _ in range(niter):
        u = A(v) - alpha * u; beta = np.linalg.norm(u); u /= beta
        v = At(u) - beta * v; alpha = np.linalg.norm(v); v /= alpha
        alphahat = np.hypot(alphabar, lmbda)
        rhopre = rho; rho = np.hypot(alphahat, beta); c, s = alphahat / rho, beta / rho
        theta = s * alpha; alphabar = c * alpha
        thetabar = sbar * rho; rhobarpre = rhobar; rhobar = np.hypot(cbar * rho, theta)
        cbar = cbar * rho / rhobar; sbar = theta / rhobar
        zeta = cbar * zetabar; zetabar = -sbar * zetabar
        hbar = h - (thetabar * rho / (rhopre * rhobarpre)) * hbar
        step = zeta / (rho * rhobar)
        x += step * hbar
        h = v - (theta / rho) * h
        rn = np.linalg.norm(b - A(x))
        if res and rn > res[-1]:
            x -= step * hbar
            break
        res.append(rn)
    return x.astype(np.float32), np.asarray(res)


def cgls(proj, geo, angles, niter):
    """CGLS of krylov_subspace_algorithms.py:39-97 with FP64 vectors over the oracle pair."""
    b = np.asarray(proj, dtype=np.float64)
    x = np.zeros(tuple(int(v) for v in geo.nVoxel), dtype=np.float64)
    r = b.copy()
    p = atb(r.astype(np.float32), geo, angles, "matched").astype(np.float64)
    gamma = float((p * p).sum())
    res = []
    for _ in range(niter):
        q = ax(p.astype(np.float32), geo, angles, "Siddon").astype(np.float64)
        alpha = gamma / float((q * q).sum())
        x += alpha * p
        r -= alpha * q
        rn = float(np.sqrt((r * r).sum()))
        if res and rn > res[-1]:
            x -= alpha * p
            break
        res.append(rn)
        s = atb(r.astype(np.float32), geo, angles, "matched").astype(np.float64)
        g1 = float((s * s).sum())
        p = s + (g1 / gamma) * p
        gamma = g1
    return x.astype(np.float32), np.asarray(res)
