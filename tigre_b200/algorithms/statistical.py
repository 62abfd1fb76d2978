"""MLEM, device-resident (Python/tigre/algorithms/statistical_algorithms.py:11-55).

    W = Atb_matched(1);  W[W <= 0] = inf;  x = 1 (no init) ;  x[x < 0] = 0
    repeat: den = Ax_interpolated(x); den[den == 0] = inf
            x *= Atb_matched(b / den) / W;  x[x < 0] = 0

Interpolated forward projector and matched backprojector as the reference; the ratio,
sensitivity division and clip are elementwise on the device.
"""
from __future__ import annotations

import numpy as np

from .. import projectors as P
from ._common import Problem, torch


def mlem_device(prob: Problem, niter, x0=None, computel2=False):
    T = torch()
    plan = prob.plan
    if x0 is None:
        x = prob.zeros_vol() + 1.0
    else:
        x = prob.to_device_vol(x0).clone()
    W = P.atb(T.ones_like(prob.b), plan, "matched")
    W[W <= 0.0] = float("inf")
    x.clamp_(min=0.0)
    den = T.empty_like(prob.b)
    img = T.empty_like(x)
    l2 = []
    for _ in range(niter):
        P.ax(x, plan, "interpolated", out=den)
        den[den == 0.0] = float("inf")
        ratio = (prob.b / den).contiguous()
        P.atb(ratio, plan, "matched", out=img)
        x.mul_(img / W).clamp_(min=0.0)
        if computel2:
            l2.append(float(P.sumsq(prob.b - P.ax(x, plan, "Siddon")).sqrt().item()))
    return x, np.asarray(l2, dtype=np.float32)


def mlem(proj, geo, angles, niter, **kwargs):
    """Drop-in for tigre.algorithms.mlem(proj, geo, angles, niter, init=, computel2=, gpuids=)."""
    prob = Problem(proj, geo, angles, kwargs.get("gpuids"))
    init = kwargs.get("init", None)
    x0 = None
    if isinstance(init, str):
        if init == "FDK":
            from .single_pass import fdk_device
            x0 = fdk_device(prob).clamp_(min=0)
        elif init != "none":
            raise ValueError("wrong value for initialization")
    elif init is not None:
        x0 = init
    x, l2 = mlem_device(prob, niter, x0, kwargs.get("computel2", False))
    out = prob.out(x)
    if kwargs.get("computel2", False):
        return out, l2.reshape(1, -1)
    return out
