"""FISTA and ISTA with TV proximal steps, device-resident (Python/tigre/algorithms/
ista_algorithms.py:13-212).

One iteration, as the reference (one block holding every view):
    x += (2/L) A^T (b - A x)        A: interpolated projector, A^T: matched backprojector (:133-150)
    x = max(x, 0)                   (noneg, iterative_recon_alg.py:344-345)
FISTA then  z = im3ddenoise(x, tviter, 1 / (2 tvlambda / L));  t' = (p + sqrt(q + 4 t^2)) / 2;
            x = z + (t - 1)/t' (z - z_prev)                     (:160-176)
ISTA:       x = im3ddenoise(x, 20, 1 / (2 * 0.1 / L))          (:190-206; the reference fixes
                                                               its lambda at 0.1)
Defaults as the reference: hyper L = 2e8, tviter 20, tvlambda 0.1, fista_p = fista_q = 1.
Extension: computel2 returns |b - A x| per iteration (the reference returns its unfilled zeros).
"""
from __future__ import annotations

import numpy as np

from .. import projectors as P
from ..utilities.im_3d_denoise import im3ddenoise
from ._common import Problem
from .krylov import _norm


def _init(prob, init):
    if isinstance(init, str):
        if init == "FDK":
            from .single_pass import fdk_device
            return fdk_device(prob).clamp_(min=0)
        if init != "none":
            raise ValueError("wrong value for initialization")
        return prob.zeros_vol()
    if init is None:
        return prob.zeros_vol()
    return prob.to_device_vol(init)


def _data_step(prob, x, step, noneg):
    r = prob.b - P.ax(x, prob.plan, "interpolated")
    x.add_(P.atb(r, prob.plan, "matched"), alpha=step)
    if noneg:
        x.clamp_(min=0)
    return x


def fista_device(prob: Problem, niter, x0=None, hyper=2.0e8, tviter=20, tvlambda=0.1, fista_p=1.0, fista_q=1.0,
                 noneg=True, computel2=False):
    bm = 1.0 / float(hyper)
    x = prob.zeros_vol() if x0 is None else x0
    x_rec = x.clone()
    lam_tv = 2.0 * bm * float(tvlambda)
    t = 1.0
    l2 = []
    for _ in range(int(niter)):
        _data_step(prob, x, 2.0 * bm, noneg)
        x_rec_old = x_rec
        x_rec = im3ddenoise(x, int(tviter), 1.0 / lam_tv)
        t_old = t
        t = (float(fista_p) + np.sqrt(float(fista_q) + 4.0 * t * t)) / 2.0
        x = x_rec + ((t_old - 1.0) / t) * (x_rec - x_rec_old)
        if computel2:
            l2.append(_norm(prob.b - P.ax(x, prob.plan, "interpolated")))
    return x, np.asarray(l2, dtype=np.float64)


def ista_device(prob: Problem, niter, x0=None, hyper=2.0e8, noneg=True, computel2=False):
    bm = 1.0 / float(hyper)
    x = prob.zeros_vol() if x0 is None else x0
    lam_tv = 2.0 * bm * 0.1
    l2 = []
    for _ in range(int(niter)):
        _data_step(prob, x, 2.0 * bm, noneg)
        x = im3ddenoise(x, 20, 1.0 / lam_tv)
        if computel2:
            l2.append(_norm(prob.b - P.ax(x, prob.plan, "interpolated")))
    return x, np.asarray(l2, dtype=np.float64)


def _entry(fn, proj, geo, angles, niter, kwargs, **extra):
    prob = Problem(proj, geo, angles, kwargs.get("gpuids"))
    x0 = _init(prob, kwargs.get("init", None))
    cl2 = bool(kwargs.get("computel2", False))
    x, l2 = fn(prob, niter, x0=x0, hyper=kwargs.get("hyper", 2.0e8), noneg=kwargs.get("noneg", True), computel2=cl2,
               **extra)
    out = prob.out(x)
    return (out, l2.reshape(1, -1).astype(np.float32)) if cl2 else out


def fista(proj, geo, angles, niter, **kwargs):
    """Drop-in for tigre.algorithms.fista(proj, geo, angles, niter, hyper=, tviter=, tvlambda=,
    fista_p=, fista_q=, init=, noneg=, computel2=, gpuids=)."""
    return _entry(fista_device, proj, geo, angles, niter, kwargs, tviter=kwargs.get("tviter", 20),
                  tvlambda=kwargs.get("tvlambda", 0.1), fista_p=kwargs.get("fista_p", 1),
                  fista_q=kwargs.get("fista_q", 1))


def ista(proj, geo, angles, niter, **kwargs):
    """Drop-in for tigre.algorithms.ista(proj, geo, angles, niter, hyper=, init=, noneg=, computel2=, gpuids=)."""
    return _entry(ista_device, proj, geo, angles, niter, kwargs)


FISTA = fista
ISTA = ista
