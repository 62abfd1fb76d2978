"""POCS-family algorithms, device-resident (Python/tigre/algorithms/pocs_algorithms.py).

ASD-POCS family (initASD_POCS.run_main_iter, :126-169; initPICCS, :187-344): per outer
iteration a SART/OS-SART sweep (FDK backprojector, nonneg), then `tviter` steps of the
regulariser with step dtvg, under the reference's adaptive rules: dtvg = alpha * |dp| after
the first sweep, reduced by alpha_red when the TV step overshoots (|dg| > rmax |dp| and the
data error exceeds epsilon), beta reduced by beta_red each iteration, and the stop criteria
(c < -0.99 and dd <= epsilon) or beta < 0.005 or n_iter >= niter.

PCSD family (initPCSD.run_main_iter, :486-560): the data sweep only while |A x - b|^2 >
epsilon, and the TV step dtvg = |A x - b| / |A x_1 - b| (1 at the first iteration, where x_1
is the image before the first regularisation); stop on the same c / beta rule or n_iter >
niter.

Regularisers: minimizeTV (POCS-TV, tigre_tv_pocs), minimizeAwTV (adaptive weights,
tigre_tv_aw_pocs, delta default -0.005) and minimizeTV_prior (PICCS, tigre_tv_piccs with
prior_ratio default 0.2), as iterative_recon_alg.py:347-360 binds them.

epsilon defaults to 0.2 |A FDK(b) - b| (maxl2err).  Everything stays on the device; the
scalars of the adaptive rules are FP64 norms read back once per iteration.
"""
from __future__ import annotations

import numpy as np

from .. import projectors as P
from .art import ART
from ._common import Problem, torch


def _norm(t):
    return float(P.sumsq(t).sqrt().item())


def _data_err(prob, x):
    return _norm(P.ax(x, prob.plan, "Siddon") - prob.b)


def _init_image(prob, kwargs):
    init = kwargs.get("init", None)
    if isinstance(init, str):
        if init == "FDK":
            from .single_pass import fdk_device
            return fdk_device(prob).clamp_(min=0)
        if init == "none":
            return prob.zeros_vol()
        raise ValueError("wrong value for initialization")
    if init is not None:
        if tuple(np.shape(init)) != tuple(int(v) for v in prob.geo.nVoxel):
            raise ValueError("wrong dimension of array for initialization")
        return prob.to_device_vol(init)
    return prob.zeros_vol()


def _epsilon(prob, kwargs):
    if "maxl2err" in kwargs:
        return float(kwargs["maxl2err"])
    from .single_pass import fdk_device
    return _data_err(prob, fdk_device(prob)) * 0.2


class _Regulariser:
    """minimizeTV / minimizeAwTV / minimizeTV_prior on a device volume, in place."""

    def __init__(self, prob, kind, tviter, kwargs):
        T = torch()
        self.kind = kind
        self.tviter = int(tviter)
        self.delta = float(kwargs.get("delta", np.float32(-0.005)))
        self.ratio = float(kwargs.get("prior_ratio", 0.2))
        self.prior = None
        if kind == "prior":
            if "prior" not in kwargs:
                raise KeyError("prior")   # the reference reads kwargs["prior"] (pocs_algorithms.py:297)
            self.prior = prob.to_device_vol(kwargs["prior"]).contiguous()
        self.work = None
        self._T = T

    def __call__(self, x, dtvg):
        if self.work is None:
            self.work = self._T.empty_like(x)
        if self.kind == "tv":
            P.tv_pocs_(x, dtvg, self.tviter, self.work)
        elif self.kind == "aw":
            P.tv_aw_pocs_(x, dtvg, self.tviter, self.delta, self.work)
        else:
            P.tv_piccs_(x, self.prior, dtvg, self.ratio, self.tviter, self.work)
        return x


def _asd_family(proj, geo, angles, niter, kwargs, blocksize, kind):
    prob = Problem(proj, geo, angles, kwargs.get("gpuids"))
    verbose = kwargs.get("verbose", False)
    art = ART(prob, blocksize, kwargs.get("OrderStrategy"), kwargs.get("lmbda", 1.0), kwargs.get("noneg", True), None,
              verbose)
    alpha = kwargs.get("alpha", 0.002)
    alpha_red = kwargs.get("alpha_red", 0.95)
    rmax = kwargs.get("rmax", 0.95)
    reg = _Regulariser(prob, kind, kwargs.get("tviter", 20), kwargs)
    beta = kwargs.get("lmbda", 1.0)
    beta_red = kwargs.get("lmbda_red", 1.0)
    epsilon = _epsilon(prob, kwargs)
    x = _init_image(prob, kwargs)
    n_iter = 0
    dtvg = None
    while True:
        x_prev = x.clone()
        art.sweep(x)
        n_iter += 1
        dd = _data_err(prob, x)
        dp_vec = x - x_prev
        dp = _norm(dp_vec)
        if n_iter == 1:
            dtvg = alpha * dp
        x_prev.copy_(x)
        reg(x, dtvg)
        dg_vec = x - x_prev
        dg = _norm(dg_vec)
        if dg > rmax * dp and dd > epsilon:
            dtvg *= alpha_red
        beta *= beta_red
        c = float((dg_vec.double() * dp_vec.double()).sum().item()) / max(dg * dp, 1e-6)
        if (c < -0.99 and dd <= epsilon) or beta < 0.005 or n_iter >= niter:
            if verbose:
                print("Stop criteria met: c=%g beta=%g iter=%d" % (c, beta, n_iter))
            break
    return prob.out(x)


def _pcsd_family(proj, geo, angles, niter, kwargs, blocksize, kind):
    prob = Problem(proj, geo, angles, kwargs.get("gpuids"))
    verbose = kwargs.get("verbose", False)
    art = ART(prob, blocksize, kwargs.get("OrderStrategy"), kwargs.get("lmbda", 1.0), kwargs.get("noneg", True), None,
              verbose)
    reg = _Regulariser(prob, kind, kwargs.get("tviter", 20), kwargs)
    beta = kwargs.get("lmbda", 1.0)
    beta_red = kwargs.get("lmbda_red", 1.0)
    epsilon = _epsilon(prob, kwargs)
    x = _init_image(prob, kwargs)
    n_iter = 0
    d_p_1st = None
    while True:
        x_prev = x.clone()
        n_iter += 1
        d_p = _data_err(prob, x)
        if d_p ** 2 > epsilon:
            art.sweep(x)
        dd = _data_err(prob, x)
        dp_vec = x - x_prev
        dp = _norm(dp_vec)
        dtvg = 1.0 if n_iter == 1 else d_p / d_p_1st
        x_prev.copy_(x)
        reg(x, dtvg)
        dg_vec = x - x_prev
        dg = _norm(dg_vec)
        if n_iter == 1:
            d_p_1st = _data_err(prob, x_prev)
        beta *= beta_red
        c = float((dg_vec.double() * dp_vec.double()).sum().item()) / max(dg * dp, 1e-6)
        if (c < -0.99 and dd <= epsilon) or beta < 0.005 or n_iter > niter:
            if verbose:
                print("Stop criteria met: c=%g beta=%g iter=%d" % (c, beta, n_iter))
            break
    return prob.out(x)


def _single_block(kwargs):
    if kwargs.get("blocksize", 1) > 1:
        print("Warning: blocksize is set to 1, please use an OS version of the algorithm for blocksize > 1")
    return 1


def asd_pocs(proj, geo, angles, niter, **kwargs):
    """ASD-POCS (pocs_algorithms.py:172-184): SART + POCS-TV."""
    return _asd_family(proj, geo, angles, niter, kwargs, _single_block(kwargs), "tv")


def awasd_pocs(proj, geo, angles, niter, **kwargs):
    """AwASD-POCS (pocs_algorithms.py:376-393): SART + adaptive-weighted TV (delta, default -0.005)."""
    return _asd_family(proj, geo, angles, niter, kwargs, _single_block(kwargs), "aw")


def os_asd_pocs(proj, geo, angles, niter, **kwargs):
    """OS-ASD-POCS (pocs_algorithms.py:396-408): OS-SART (blocksize default 20) + POCS-TV."""
    return _asd_family(proj, geo, angles, niter, kwargs, kwargs.get("blocksize", 20), "tv")


def os_awasd_pocs(proj, geo, angles, niter, **kwargs):
    """OS-AwASD-POCS (pocs_algorithms.py:411-431): OS-SART + adaptive-weighted TV."""
    return _asd_family(proj, geo, angles, niter, kwargs, kwargs.get("blocksize", 20), "aw")


def piccs(proj, geo, angles, niter, **kwargs):
    """PICCS (pocs_algorithms.py:346-358): SART + prior TV (prior=, prior_ratio default 0.2)."""
    return _asd_family(proj, geo, angles, niter, kwargs, _single_block(kwargs), "prior")


def os_piccs(proj, geo, angles, niter, **kwargs):
    """OS-PICCS (pocs_algorithms.py:361-373): OS-SART (blocksize default 20) + prior TV."""
    return _asd_family(proj, geo, angles, niter, kwargs, kwargs.get("blocksize", 20), "prior")


def pcsd(proj, geo, angles, niter, **kwargs):
    """PCSD (pocs_algorithms.py:573-586): data sweep while |Ax-b|^2 > epsilon, TV step |Ax-b|/|Ax_1-b|."""
    return _pcsd_family(proj, geo, angles, niter, kwargs, _single_block(kwargs), "tv")


def aw_pcsd(proj, geo, angles, niter, **kwargs):
    """AwPCSD (pocs_algorithms.py:589-608): PCSD with adaptive-weighted TV."""
    return _pcsd_family(proj, geo, angles, niter, kwargs, _single_block(kwargs), "aw")


def os_pcsd(proj, geo, angles, niter, **kwargs):
    """OS-PCSD (pocs_algorithms.py:611-625): PCSD with OS-SART (blocksize default 20)."""
    return _pcsd_family(proj, geo, angles, niter, kwargs, kwargs.get("blocksize", 20), "tv")


def os_aw_pcsd(proj, geo, angles, niter, **kwargs):
    """OS-AwPCSD (pocs_algorithms.py:628-648): PCSD with OS-SART and adaptive-weighted TV."""
    return _pcsd_family(proj, geo, angles, niter, kwargs, kwargs.get("blocksize", 20), "aw")
