"""SART family (OS-SART, SIRT, SART), device-resident.

Same algorithm as the reference's IterativeReconAlg
(Python/tigre/algorithms/iterative_recon_alg.py:131-401, art_family_algorithms.py):

    W = 1 / A(ones) on a 2^3 box enlarged to the detector (set_w, :214-230)
    V_j = mean_z A_j^T(ones) (FDK backprojector, shrunk box) per subset (set_v, :232-270)
    per subset j:  x += lambda / V_j * A_j^T_FDK( W_j * (b_j - A_j x) );  x = max(x, 0)

Per subset the forward projection, the weighted residual, the FDK
backprojection and the update run on the GPU; subsets that are contiguous
view ranges reuse the full plan (angle_range), others get their own plan.
Storage precision (extension): storage=torch.bfloat16/float16 keeps the
volume and the projections in that type (FP32 arithmetic, FP64 geometry);
proj_storage= overrides the projections' type alone (torch.float32 keeps
them exact); rounding="stochastic" (with seed=) rounds each volume update stochastically
instead of to nearest, so updates below half a unit in the last place are
kept in expectation.  The volume update itself is one fused kernel
(tigre_sart_update).
"""
from __future__ import annotations

import copy

import numpy as np

from .. import _native as N
from .. import projectors as P
from ..utilities.order_subsets import order_subsets
from ..utilities.Measure_Quality import QualityLog
from ._common import Problem, torch


class ART:
    def __init__(self, prob: Problem, blocksize, order=None, lmbda=1.0, noneg=True, storage=None, verbose=False,
                 rounding="nearest", seed=0, proj_storage=None):
        T = torch()
        proj_storage = storage if proj_storage is None else proj_storage
        self.prob = prob
        self.rounding = rounding
        self.seed = int(seed)
        self.step = 0
        self.lmbda = float(lmbda)
        self.noneg = noneg
        self.verbose = verbose
        self.storage = storage or T.float32
        g = prob.geo
        self.blocks, self.index = order_subsets(prob.angles, blocksize, order)
        self.index = [np.asarray(i).reshape(-1).astype(np.int64) for i in self.index]
        self.W = self._weights_w()
        self.V = self._weights_v()
        self.plans = []
        for idx in self.index:
            rng = prob.contiguous_range(idx)
            if rng is not None:
                self.plans.append((prob.plan, rng))
            else:
                sub = prob.sub_geometry(idx)
                self.plans.append((N.get_plan(N.checked_geometry(sub, sub.angles), prob.device.index), None))
        self.b = prob.b.to(proj_storage) if proj_storage not in (None, T.float32) else prob.b

    def _weights_w(self):
        T = torch()
        prob = self.prob
        gx = copy.deepcopy(prob.geo_full)
        gx.sVoxel = np.array(gx.sVoxel, dtype=np.float64)
        gx.sVoxel[1:] = gx.sVoxel[1:] * 1.1
        gx.sVoxel[0] = max(float(gx.sDetector[0]), gx.sVoxel[0])
        gx.nVoxel = np.array([2, 2, 2])
        gx.dVoxel = gx.sVoxel / gx.nVoxel
        plan = N.get_plan(N.checked_geometry(gx, prob.angles), prob.device.index)
        W = P.ax(T.ones((2, 2, 2), dtype=T.float32, device=prob.device), plan, "Siddon")
        W[W <= float(min(np.asarray(prob.geo_full.dVoxel, dtype=np.float64) / 2))] = float("inf")
        return 1.0 / W

    def _weights_v(self):
        T = torch()
        prob = self.prob
        g = prob.geo
        V = []
        for idx in self.index:
            if getattr(g, "mode", "cone") == "parallel":   # set_v: V = block length (:265-266)
                V.append(T.full(tuple(int(v) for v in g.nVoxel[1:]), float(len(idx)), dtype=T.float32,
                                device=prob.device))
                continue
            gx = prob.sub_geometry(idx)
            sv = np.array(gx.sVoxel, dtype=np.float64)
            gx.sVoxel = sv * np.max(sv[1:] / np.linalg.norm(sv[1:])) * 0.9
            gx.dVoxel = gx.sVoxel / gx.nVoxel
            plan = N.get_plan(N.checked_geometry(gx, gx.angles), prob.device.index)
            ones = T.ones((len(idx),) + tuple(int(v) for v in g.nDetector), dtype=T.float32, device=prob.device)
            v = P.atb(ones, plan, "FDK").mean(dim=0)
            v[v == 0.0] = float("inf")
            V.append(v.contiguous())
        return V

    def sweep(self, x):
        """One pass over all subsets (art_data_minimizing)."""
        T = torch()
        for j, idx in enumerate(self.index):
            plan, rng = self.plans[j]
            if rng is not None:
                b_j = self.b[rng[0]:rng[1]]
                w_j = self.W[rng[0]:rng[1]]
                est = P.ax(x, plan, "Siddon", angle_range=rng, out_dtype=T.float32)
            else:
                ii = T.as_tensor(idx, device=x.device)
                b_j = self.b.index_select(0, ii)
                w_j = self.W.index_select(0, ii)
                est = P.ax(x, plan, "Siddon", out_dtype=T.float32)
            err = (w_j * (b_j.float() - est)).contiguous()
            bp = P.atb(err, plan, "FDK", angle_range=rng, out_dtype=T.float32)
            P.sart_update_(x, bp, self.V[j], self.lmbda, self.noneg, self.rounding, self.seed, self.step)
            self.step += 1
        return x


def _run(proj, geo, angles, niter, blocksize, kwargs):
    prob = Problem(proj, geo, angles, kwargs.get("gpuids"))
    T = torch()
    storage = kwargs.get("storage", None)
    art = ART(prob, blocksize, kwargs.get("OrderStrategy"), kwargs.get("lmbda", 1.0), kwargs.get("noneg", True),
              storage, kwargs.get("verbose", False), kwargs.get("rounding", "nearest"), kwargs.get("seed", 0),
              kwargs.get("proj_storage"))
    init = kwargs.get("init", None)
    if isinstance(init, str) and init == "FDK":
        from .single_pass import fdk_device
        x = fdk_device(prob).clamp_(min=0)
    elif init is not None and not isinstance(init, str):
        x = prob.to_device_vol(init)
    else:
        x = prob.zeros_vol()
    if storage is not None and storage != T.float32:
        x = x.to(storage)
    l2 = []
    callback = kwargs.get("callback")
    quality = QualityLog(kwargs.get("Quameasopts"), niter)
    for it in range(niter):
        quality.before(x)
        art.sweep(x)
        if kwargs.get("computel2", False):
            l2.append(float(T.linalg.vector_norm((prob.b - P.ax(x, prob.plan, "Siddon", out_dtype=T.float32))
                                                 .double()).item()))
        quality.after(x, it)
        if callback is not None:
            callback(it, x)
    out = prob.out(x.float() if x.dtype != T.float32 else x)
    if kwargs.get("computel2", False) and not quality.active:
        return out, np.asarray(l2, dtype=np.float32).reshape(1, -1)
    if quality.active:
        return out, quality.errors(l2 if kwargs.get("computel2", False) else None)
    return out


def ossart(proj, geo, angles, niter, **kwargs):
    """Drop-in for tigre.algorithms.ossart (blocksize default 20)."""
    return _run(proj, geo, angles, niter, kwargs.pop("blocksize", 20), kwargs)


def sirt(proj, geo, angles, niter, **kwargs):
    kwargs.pop("blocksize", None)
    return _run(proj, geo, angles, niter, len(np.atleast_1d(angles)), kwargs)


def sart(proj, geo, angles, niter, **kwargs):
    kwargs.pop("blocksize", None)
    return _run(proj, geo, angles, niter, 1, kwargs)


def _run_tv(proj, geo, angles, niter, blocksize, kwargs):
    """SART_TV / OSSART_TV (art_family_algorithms.py:65-152): per iteration one (OS-)SART sweep,
    then im3ddenoise(res, tviter, tvlambda) (TV proximal operator on the device)."""
    from ..utilities.im_3d_denoise import im3ddenoise
    prob = Problem(proj, geo, angles, kwargs.get("gpuids"))
    art = ART(prob, blocksize, kwargs.get("OrderStrategy"), kwargs.get("lmbda", 1.0), kwargs.get("noneg", True), None,
              kwargs.get("verbose", False))
    tvlambda = kwargs.get("tvlambda", 50)
    tviter = kwargs.get("tviter", 50)
    init = kwargs.get("init", None)
    if isinstance(init, str) and init == "FDK":
        from .single_pass import fdk_device
        x = fdk_device(prob).clamp_(min=0)
    elif init is not None and not isinstance(init, str):
        x = prob.to_device_vol(init)
    else:
        x = prob.zeros_vol()
    for _ in range(niter):
        art.sweep(x)
        x = im3ddenoise(x, tviter, tvlambda).contiguous()
    return prob.out(x)


def sart_tv(proj, geo, angles, niter, **kwargs):
    """Drop-in for tigre.algorithms.sart_tv (blocksize 1, tvlambda 50, tviter 50)."""
    if kwargs.get("blocksize", 1) > 1:
        print("Warning: blocksize is set to 1, please use an OS version of the algorithm for blocksize > 1")
    return _run_tv(proj, geo, angles, niter, 1, kwargs)


def ossart_tv(proj, geo, angles, niter, **kwargs):
    """Drop-in for tigre.algorithms.ossart_tv (blocksize default 20, tvlambda 50, tviter 50)."""
    return _run_tv(proj, geo, angles, niter, kwargs.get("blocksize", 20), kwargs)
