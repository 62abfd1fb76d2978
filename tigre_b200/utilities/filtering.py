"""FDK pre-processing on the device: cosine weights, Parker weights, ramp filtering.

Same filter construction as the reference (Python/tigre/utilities/filtering.py:15-94):
filter length max(64, 2^nextpow2(2 nU)), spatial ramp kernel ramp_flat(n), window
(ram_lak / shepp_logan / cosine / hamming / hann) applied to |FFT(kernel)|*2,
rows zero-padded to the filter length and centred, result scaled by
(DSD/DSO) (2 pi / nangles) / (4 dU).  The reference filters on the host with
scipy.fft, two projections per complex FFT; here all rows of all views are
filtered on the device in one batched real FFT (cuFFT through torch.fft), in
float64 arithmetic when precision="float64" (default float32, like scipy on
complex64).

Parker weights: Wesarg et al., "Parker weights revisited", Med. Phys. 29(3), 2002
(Python/tigre/utilities/parkerweight.py:23-78).  The Python reference never
enables them in FDK (single_pass_algorithms.py:199 passes parker=False); the
MATLAB front end does for short scans (MATLAB/Algorithms/FDK.m:153-161).
"""
from __future__ import annotations

import warnings

import numpy as np


def nextpow2(n):
    i = 1
    while (2 ** i) <= n:
        i += 1
    return i


def ramp_flat(n):
    nn = np.arange(-n / 2, n / 2)
    h = np.zeros(nn.shape, dtype=np.float32)
    h[int(n / 2)] = 1 / 4
    odd = nn % 2 == 1
    h[odd] = -1 / (np.pi * nn[odd]) ** 2
    return h, nn


def filter_kernel(filter, kernel, order, d=1, verbose=False):  # noqa: A002
    f_kernel = abs(np.fft.fft(kernel)) * 2
    filt = f_kernel[: int((order / 2) + 1)]
    w = 2 * np.pi * np.arange(len(filt)) / order
    if filter in {"ram_lak", None}:
        if filter is None and verbose:
            warnings.warn("no filter selected, using default ram_lak")
    elif filter == "shepp_logan":
        filt[1:] *= np.sin(w[1:] / (2 * d)) / (w[1:] / (2 * d))
    elif filter == "cosine":
        filt[1:] *= np.cos(w[1:] / (2 * d))
    elif filter == "hamming":
        filt[1:] *= 0.54 + 0.46 * np.cos(w[1:] / d)
    elif filter == "hann":
        filt[1:] *= (1 + np.cos(w[1:] / d)) / 2
    else:
        raise ValueError("filter not recognized: " + str(filter))
    filt[w > np.pi * d] = 0
    filt = np.hstack((filt, filt[1:-1][::-1]))
    return filt.astype(np.float32)


def ramp_response(nU, filter=None):  # noqa: A002,N803
    """(filter length, full-length frequency response) of the reference's ramp filter."""
    L = max(64, 2 ** nextpow2(2 * nU))
    return L, filter_kernel(filter, ramp_flat(L)[0], L)


def filter_projections(proj, geo, nangles, filter=None, precision="float32", angular_weight=None):  # noqa: A002
    """Ramp-filter device projections (n, nV, nU); returns a new tensor.  angular_weight
    replaces 2 pi / nangles (short scans with Parker weights use 2 * mean view step,
    MATLAB/Utilities/filtering.m:47-48)."""
    import torch
    nU = proj.shape[-1]
    L, filt = ramp_response(nU, filter)
    pad = int((L - nU) // 2)
    dsd = float(np.asarray(geo.DSD).reshape(-1)[0])
    dso = float(np.asarray(geo.DSO).reshape(-1)[0])
    aw = (2 * np.pi / nangles) if angular_weight is None else float(angular_weight)
    scale = (dsd / dso) * aw / (4 * float(geo.dDetector[1]))
    cdt = torch.float64 if precision == "float64" else torch.float32
    H = torch.from_numpy(filt[: L // 2 + 1].astype(np.float64)).to(device=proj.device, dtype=cdt)
    buf = torch.zeros(proj.shape[:-1] + (L,), dtype=cdt, device=proj.device)
    buf[..., pad:pad + nU] = proj.to(cdt)
    spec = torch.fft.rfft(buf, dim=-1)
    spec *= H
    out = torch.fft.irfft(spec, n=L, dim=-1)[..., pad:pad + nU]
    return (out * scale).to(torch.float32).contiguous()


def cosine_weights(geo, device=None):
    """DSD / sqrt(DSD^2 + u^2 + v^2) on the detector grid (single_pass_algorithms.py:186-197)."""
    nv, nu = int(geo.nDetector[0]), int(geo.nDetector[1])
    xv = np.arange(-nu / 2 + 0.5, 1 + nu / 2 - 0.5) * float(geo.dDetector[1])
    yv = np.arange(-nv / 2 + 0.5, 1 + nv / 2 - 0.5) * float(geo.dDetector[0])
    yy, xx = np.meshgrid(xv, yv)
    dsd = float(np.asarray(geo.DSD).reshape(-1)[0])
    w = dsd / np.sqrt(dsd ** 2 + xx ** 2 + yy ** 2)
    if device is None:
        return w.astype(np.float32)
    import torch
    return torch.from_numpy(w.astype(np.float32)).to(device)


def _s_function(b):
    w = np.zeros(b.shape)
    w[b <= -0.5] = 0
    m = np.abs(b) < 0.5
    w[m] = 0.5 * (1 + np.sin(np.pi * b[m]))
    w[b >= 0.5] = 1
    return w


def parker_weights(geo, angles, q=1.0):
    """(nangles, nU) Parker weights (parkerweight.py:23-78; axis and flip of ParkerWeight.m)."""
    angles = np.asarray(angles, dtype=np.float64)
    if angles.ndim == 2:
        angles = angles[:, 0]
    nu, ddu = int(geo.nDetector[1]), float(geo.dDetector[1])
    alpha = np.arctan((np.arange(nu) - nu / 2 + 0.5) * ddu / np.mean(geo.DSD))
    # weights run along u; flipped for increasing angles (MATLAB/Utilities/ParkerWeight.m:12-15 --
    # the Python port indexes the v extent and only works for square detectors)
    if np.all(np.diff(angles) >= 0):
        alpha = -alpha
    delta = abs(alpha[0] - alpha[-1]) / 2
    totangles = abs(angles[0] - angles[-1])
    if totangles > 2 * np.pi:
        warnings.warn("Computing Parker weights for scanning angle equal or bigger than 2*pi "
                      "Consider disabling Parker weights.")
    if totangles < np.pi + 2 * delta:
        warnings.warn("Scanning angles smaller than pi+cone_angle. This is limited angle tomography, \n"
                      "there is no sufficient data, thus weighting for data redundancy is not required.")
    eps = max(totangles - (np.pi + 2 * delta), 0)

    def b(a):
        return q * (2 * delta - 2 * a + eps)

    W = np.empty((angles.shape[0], alpha.shape[0]))
    for i in range(angles.shape[0]):
        beta = abs(angles[i] - angles[0])
        W[i] = 0.5 * (_s_function(beta / b(alpha) - 0.5)
                      + _s_function((beta - 2 * delta + 2 * alpha - eps) / b(alpha) + 0.5)
                      - _s_function((beta - np.pi + 2 * alpha) / b(-alpha) - 0.5)
                      - _s_function((beta - np.pi - 2 * delta - eps) / b(-alpha) + 0.5))
    return W.astype(np.float32)


def filtering(proj, geo, angles, parker, verbose=False):
    """Host-array mirror of tigre.utilities.filtering.filtering (same arguments)."""
    import torch
    t = torch.from_numpy(np.ascontiguousarray(proj, dtype=np.float32))
    if torch.cuda.is_available():
        t = t.cuda()
    aw = None
    if parker:
        W = torch.from_numpy(parker_weights(geo, angles, parker)).to(t.device)
        t = t * W[:, None, :]
        a = np.asarray(angles, dtype=np.float64)
        a = a[:, 0] if a.ndim == 2 else a
        aw = 2 * np.mean(np.abs(np.diff(a)))
    out = filter_projections(t, geo, len(angles), getattr(geo, "filter", None), angular_weight=aw)
    return out.cpu().numpy()
