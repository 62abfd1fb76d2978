"""ASD-POCS, device-resident (Python/tigre/algorithms/pocs_algorithms.py:15-185).

Per outer iteration: a SART sweep (blocksize 1, FDK backprojector, nonneg),
then `tviter` POCS-TV steps with step dtvg, with the reference's adaptive
rules: dtvg = alpha * |dp| after the first sweep, reduced by alpha_red when
the TV step overshoots (|dg| > rmax |dp| and the data error exceeds
epsilon), beta reduced by beta_red each iteration, and the stop criteria
(c < -0.99 and dd <= epsilon) or beta < 0.005 or n_iter >= niter.
epsilon defaults to 0.2 |A FDK(b) - b| (maxl2err).
"""
from __future__ import annotations

import numpy as np

from .. import projectors as P
from .art import ART
from ._common import Problem, torch


def asd_pocs(proj, geo, angles, niter, **kwargs):
    T = torch()
    prob = Problem(proj, geo, angles, kwargs.get("gpuids"))
    art = ART(prob, 1, kwargs.get("OrderStrategy"), kwargs.get("lmbda", 1.0), kwargs.get("noneg", True), None,
              kwargs.get("verbose", False))
    alpha = kwargs.get("alpha", 0.002)
    alpha_red = kwargs.get("alpha_red", 0.95)
    rmax = kwargs.get("rmax", 0.95)
    tviter = kwargs.get("tviter", 20)
    beta = kwargs.get("lmbda", 1.0)
    beta_red = kwargs.get("lmbda_red", 1.0)
    if "maxl2err" in kwargs:
        epsilon = float(kwargs["maxl2err"])
    else:
        from .single_pass import fdk_device
        f = fdk_device(prob)
        epsilon = float(T.linalg.vector_norm((P.ax(f, prob.plan, "Siddon") - prob.b).double()).item()) * 0.2
    x = prob.zeros_vol()
    init = kwargs.get("init", None)
    if init is not None and not isinstance(init, str):
        x = prob.to_device_vol(init)
    work = T.empty_like(x)
    n_iter = 0
    dtvg = None
    while True:
        x_prev = x.clone()
        art.sweep(x)
        n_iter += 1
        dd = float(T.linalg.vector_norm((P.ax(x, prob.plan, "Siddon") - prob.b).double()).item())
        dp_vec = x - x_prev
        dp = float(T.linalg.vector_norm(dp_vec.double()).item())
        if n_iter == 1:
            dtvg = alpha * dp
        x_prev = x.clone()
        P.tv_pocs_(x, dtvg, tviter, work)
        dg_vec = x - x_prev
        dg = float(T.linalg.vector_norm(dg_vec.double()).item())
        if dg > rmax * dp and dd > epsilon:
            dtvg *= alpha_red
        beta *= beta_red
        c = float((dg_vec.double() * dp_vec.double()).sum().item()) / max(dg * dp, 1e-6)
        if (c < -0.99 and dd <= epsilon) or beta < 0.005 or n_iter >= niter:
            if kwargs.get("verbose", False):
                print("Stop criteria met: c=%g beta=%g iter=%d" % (c, beta, n_iter))
            break
    return prob.out(x)
