"""FDK on the device (Python/tigre/algorithms/single_pass_algorithms.py:12-202).

Steps as the reference: optional detector-offset (Wang) pre-weighting with
zero padding (:78-178), cosine weights DSD/sqrt(DSD^2+u^2+v^2) (:186-197),
ramp filtering (filtering.py), FDK-weighted backprojection.  Extension:
parker=True applies Parker short-scan weights before filtering, the wiring
the MATLAB front end has (MATLAB/Algorithms/FDK.m:153-161) and the Python one
lacks.  Everything after the optional Wang step runs on the GPU.
"""
from __future__ import annotations

import copy

import numpy as np

from .. import projectors as P
from ..utilities import filtering as F
from ._common import Problem, torch


def _wang(proj, geo):
    """Zero padding + Wang pre-weighting for an offset detector (:78-178), host numpy."""
    zgeo = copy.deepcopy(geo)
    off = geo.offDetector[1, 0] if np.ndim(geo.offDetector) == 2 else geo.offDetector[1]
    padwidth = int(2 * off / geo.dDetector[1])
    zgeo.offDetector = np.array(zgeo.offDetector, dtype=np.float64)
    if zgeo.offDetector.ndim == 2:
        zgeo.offDetector[:, 1] = off - padwidth / 2 * geo.dDetector[1]
    else:
        zgeo.offDetector[1] = off - padwidth / 2 * geo.dDetector[1]
    zgeo.nDetector = np.array(zgeo.nDetector)
    zgeo.nDetector[1] = abs(padwidth) + geo.nDetector[1]
    zgeo.sDetector = np.array(zgeo.sDetector, dtype=np.float64)
    zgeo.sDetector[1] = zgeo.nDetector[1] * zgeo.dDetector[1]
    theta = (geo.sDetector[1] / 2 - abs(off)) * np.sign(off)
    pad = np.zeros((proj.shape[0], proj.shape[1], abs(padwidth)), dtype=proj.dtype)
    zproj = np.concatenate((pad, proj), axis=2) if off > 0 else np.concatenate((proj, pad), axis=2)
    cor = getattr(zgeo, "COR", 0)
    offset = np.asarray(zgeo.offDetector)[..., 1] if np.ndim(zgeo.offDetector) == 2 else zgeo.offDetector[1]
    offset = np.asarray(offset).reshape(-1)[0] + (np.asarray(zgeo.DSD).reshape(-1)[0] /
                                                  np.asarray(zgeo.DSO).reshape(-1)[0]) * np.asarray(cor).reshape(-1)[0]
    dso, dsd = np.asarray(zgeo.DSO).reshape(-1)[0], np.asarray(zgeo.DSD).reshape(-1)[0]
    us = (np.arange(-zgeo.nDetector[1] / 2 + 0.5, zgeo.nDetector[1] / 2 - 0.5 + 1) * zgeo.dDetector[1]
          + abs(offset)) * dso / dsd
    abstheta = abs(theta * dso / dsd)
    w = np.ones(zproj.shape[1:])
    for ii in range(int(zgeo.nDetector[1])):
        t = us[ii]
        if abs(t) <= abstheta:
            w[:, ii] = 0.5 * (np.sin((np.pi / 2) * np.arctan(t / dso) / np.arctan(abstheta / dso)) + 1)
        if t < -abstheta:
            w[:, ii] = 0
    if theta < 0:
        w = np.fliplr(w)
    return (zproj * w * 2).astype(np.float32), zgeo


def fdk_device(prob: Problem, filter=None, parker=False, out=None, proj=None):  # noqa: A002
    """FDK of the Problem's projections (or of `proj`, a device stack of the same geometry);
    returns a device volume."""
    T = torch()
    g = prob.geo
    w = F.cosine_weights(g, device=prob.device)
    pw = (prob.b if proj is None else proj) * w
    aw = None
    if parker:
        W = T.from_numpy(F.parker_weights(g, prob.angles, 1.0 if parker is True else float(parker))).to(prob.device)
        pw = pw * W[:, None, :]
        aw = 2 * float(np.mean(np.abs(np.diff(prob.angles[:, 0].astype(np.float64)))))
    filt = F.filter_projections(pw, g, prob.n, filter, angular_weight=aw)
    return P.atb(filt, prob.plan, "FDK", out=out)


def FDK(proj, geo, angles, **kwargs):  # noqa: N802
    """Drop-in for tigre.algorithms.fdk(proj, geo, angles, filter=, dowang=, gpuids=, verbose=) (+ parker=)."""
    dowang = kwargs.get("dowang", True)
    g0 = copy.deepcopy(geo)
    g0.check_geo(angles)
    if not np.any(g0.offDetector):
        dowang = False
    if dowang:
        host = proj.cpu().numpy() if type(proj).__module__.startswith("torch") else np.asarray(proj)
        proj, geo = _wang(host, g0)
    prob = Problem(proj, geo, angles, kwargs.get("gpuids"))
    vol = fdk_device(prob, kwargs.get("filter", None), kwargs.get("parker", False))
    return prob.out(vol)


fdk = FDK


def fbp(proj, geo, angles, **kwargs):
    """Parallel-beam FBP, drop-in for tigre.algorithms.fbp (single_pass_algorithms.py:206-228):
    ramp filter on the device, parallel backprojection, times DSO/DSD."""
    if getattr(geo, "mode", "cone") != "parallel":
        raise ValueError("Only use FBP for parallel beam. Check geo.mode.")
    prob = Problem(proj, geo, angles, kwargs.get("gpuids"))
    g = prob.geo
    filt = F.filter_projections(prob.b, g, prob.n, kwargs.get("filter", None))
    vol = P.atb(filt, prob.plan, "FDK")
    vol *= float(np.asarray(g.DSO).reshape(-1)[0]) / float(np.asarray(g.DSD).reshape(-1)[0])
    return prob.out(vol)
