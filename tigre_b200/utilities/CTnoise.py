"""Projection noise, drop-in for tigre.utilities.CTnoise (Python/tigre/utilities/CTnoise.py:4-33)
and the _RandomNumberGenerator extension (_randomNumberGenerator.pyx: add_poisson, add_noise).

The counts are drawn on the device by tigre_add_noise: Poisson(lambda) plus, for add_noise,
N(mu, sigma), from a counter-based Philox4x32-10 stream keyed by `seed`.  The reference seeds
every call with 1234, so repeated calls on the same input return the same noise; the default
seed here is 1234 for the same behaviour (its numbers differ: curand's XORWOW stream over a
fixed grid cannot be reproduced).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from .. import _native as N
from .errors import TigreCudaCallError
from .gpu import device_list

DEFAULT_SEED = 1234


def _is_cuda(x):
    return type(x).__module__.startswith("torch") and getattr(x, "is_cuda", False)


def _noise(src, gaussian, mu, sigma, gpuids, seed):
    if _is_cuda(src):
        from .. import projectors
        out = src.detach().contiguous().float().clone()
        N.check(N.lib().tigre_add_noise(C.c_void_p(out.data_ptr()), C.c_void_p(out.data_ptr()), out.numel(),
                                        int(gaussian), float(mu), float(sigma), int(seed) & (2**64 - 1),
                                        projectors._stream(out)), "tigre_add_noise")
        return out
    src = np.ascontiguousarray(src, dtype=np.float32)
    out = np.empty_like(src)
    devices = device_list(gpuids)
    ids = (C.c_int * len(devices))(*devices)
    rc = N.lib().tigre_noise_1d(src.ctypes.data, src.size, int(gaussian), float(mu), float(sigma),
                                int(seed) & (2**64 - 1), out.ctypes.data, C.cast(ids, C.c_void_p), len(devices))
    if rc:
        raise TigreCudaCallError("RandomNumberGenerator::", rc, N.last_error())
    return out


def add_poisson(src, gpuids=None, seed=DEFAULT_SEED):
    """Poisson(src) elementwise (poisson_1d)."""
    return _noise(src, 0, 0.0, 0.0, gpuids, seed)


def add_noise(poisson_lambda, gaussian_mu, gaussian_sigma, gpuids=None, seed=DEFAULT_SEED):
    """Poisson(lambda) + N(mu, sigma) elementwise (poisson_gaussian_1d)."""
    return _noise(poisson_lambda, 1, gaussian_mu, gaussian_sigma, gpuids, seed)


def add(projections, Gaussian=None, Poisson=None, seed=DEFAULT_SEED):  # noqa: N803
    """Noisy projections as CTnoise.add: counts Poisson * exp(-p / max p), Poisson and Gaussian
    noise on them, then back to line integrals.  Poisson defaults to ceil(log2(max |p|)) and
    Gaussian to [0, 0.5], as in the reference (CTnoise.py:7-22)."""
    if Poisson is not None:
        if not np.isscalar(Poisson):
            raise ValueError("Poisson value should be an scalar, is " + str(type(Poisson)) + " instead.")
    if Gaussian is not None:
        if not isinstance(Gaussian, np.ndarray):
            raise ValueError("Gaussian value should be an array, is " + str(type(Gaussian)) + " instead.")
        if Gaussian.shape != (2,):
            raise ValueError("Gaussian shape should be 1x2, is " + str(Gaussian.shape) + "instead.")
    else:
        Gaussian = np.array([0, 0.5])
    if _is_cuda(projections):
        import torch
        p = projections.detach().float()
        if Poisson is None:
            Poisson = float(np.ceil(np.log2(float(p.abs().max().item()))))
        max_proj = float(p.max().item())
        # counts in FP64, rounded once to FP32, on both paths
        lam = (float(Poisson) * torch.exp(-p.double() / max_proj)).float().contiguous()
        noisy = add_noise(lam, float(Gaussian[0]), float(Gaussian[1]), seed=seed)
        return (-torch.log(noisy / float(Poisson)) * max_proj).float()
    projections = np.asarray(projections)
    if Poisson is None:
        Poisson = np.ceil(np.log2(np.max(np.abs(projections))))
    max_proj = np.max(projections)
    lam = float(Poisson) * np.exp(-np.asarray(projections, dtype=np.float64) / float(max_proj))
    noisy = add_noise(lam.astype(np.float32), float(Gaussian[0]), float(Gaussian[1]), seed=seed)
    return np.float32(-np.log(noisy / Poisson) * max_proj)
