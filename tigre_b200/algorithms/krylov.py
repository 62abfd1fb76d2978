"""Krylov solvers (CGLS, LSQR, LSMR), device-resident.

Same iteration and outputs as the reference (Python/tigre/algorithms/
krylov_subspace_algorithms.py:22-99): Siddon forward projection, matched
backprojection,

    r = b - A x0;  p = A^T r;  gamma = |p|^2
    repeat:  q = A p;  alpha = gamma / |q|^2;  x += alpha p;  r -= alpha q
             s = A^T r;  gamma' = |s|^2;  p = s + (gamma'/gamma) p

with the reference's divergence rule: when the residual grows, the last step
is undone and the iteration stops.  Differences in how:

* x, r, p, q, s live in HBM; alpha and beta are FP64 device scalars read by
  the fused update kernels (tigre_cgls_step / tigre_cgls_direction), so an
  iteration needs one 8-byte device->host read (the residual) and no host
  vector arithmetic;
* the logged residual is |r| from the recurrence (one Ax per iteration fewer
  than the reference's explicit |b - A x|, krylov_subspace_algorithms.py:66);
  pass true_residual=True for the explicit form;
* tol (extension): stop when |r| / |b| <= tol.
"""
from __future__ import annotations

import time

import numpy as np

from .. import projectors as P
from ._common import Problem, torch


class CGLSResult:
    def __init__(self, x, residuals, times):
        self.x = x
        self.residuals = residuals
        self.times = times


def cgls_device(prob: Problem, niter, x0=None, tol=None, true_residual=False, restart=True, verbose=False,
                callback=None):
    """Run CGLS on a Problem; returns (x tensor, residual norms, wall seconds per iteration)."""
    T = torch()
    dev = prob.device
    plan = prob.plan
    b = prob.b
    x = prob.zeros_vol() if x0 is None else prob.to_device_vol(x0)
    if x0 is None:
        r = b.clone()
    else:
        r = b - P.ax(x, plan, "Siddon")
    p = P.atb(r, plan, "matched")
    s = T.empty_like(p)
    q = T.empty_like(b)
    # device scalars: [gamma, |q|^2, gamma', |r|^2, |b|^2]
    sc = T.zeros(5, dtype=T.float64, device=dev)
    P.sumsq(p, out=sc[0])
    P.sumsq(b, out=sc[4])
    bnorm = float(sc[4].sqrt().item())
    nvol, nproj = x.numel(), r.numel()
    lib = __import__("tigre_b200._native", fromlist=["lib"]).lib()
    import ctypes as C

    def ptr(t):
        return C.c_void_p(t.data_ptr())

    stream = C.c_void_p(T.cuda.current_stream(dev).cuda_stream)
    l2 = []
    times = []
    for it in range(niter):
        t0 = time.perf_counter()
        P.ax(p, plan, "Siddon", out=q)
        sc[1].zero_()
        sc[3].zero_()
        P.sumsq(q, out=sc[1])
        # x += (gamma/|q|^2) p ; r -= (gamma/|q|^2) q ; sc[3] = |r|^2
        rc = lib.tigre_cgls_step(ptr(x), ptr(p), nvol, ptr(r), ptr(q), nproj, ptr(sc[0]), ptr(sc[1]), ptr(sc[3]),
                                 stream)
        if rc:
            raise RuntimeError("tigre_cgls_step failed")
        if true_residual:
            res = float(T.linalg.vector_norm((b - P.ax(x, plan, "Siddon")).double()).item())
        else:
            res = float(sc[3].sqrt().item())
        if it > 0 and res > l2[-1]:
            # divergence: undo the step and stop (krylov_subspace_algorithms.py:67-78)
            x.add_(p, alpha=-float((sc[0] / sc[1]).item()))
            if verbose:
                print("CGLS exited due to divergence at iteration", it)
            times.append(time.perf_counter() - t0)
            break
        l2.append(res)
        P.atb(r, plan, "matched", out=s)
        sc[2].zero_()
        P.sumsq(s, out=sc[2])
        rc = lib.tigre_cgls_direction(ptr(p), ptr(s), nvol, ptr(sc[2]), ptr(sc[0]), stream)
        if rc:
            raise RuntimeError("tigre_cgls_direction failed")
        sc[0].copy_(sc[2])
        times.append(time.perf_counter() - t0)
        if callback is not None:
            callback(it, x, res / max(bnorm, 1e-30))
        if tol is not None and res <= tol * bnorm:
            break
    return x, np.asarray(l2, dtype=np.float64), times


def cgls(proj, geo, angles, niter, **kwargs):
    """Drop-in for tigre.algorithms.cgls(proj, geo, angles, niter, **kwargs).

    Keywords as the reference: init (None | "FDK" | array), verbose, computel2,
    gpuids, restart; plus tol, true_residual, return_residuals (extensions).
    Returns the volume (numpy for numpy input), and (volume, l2 residuals)
    when computel2=True.
    """
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
    x, l2, _ = cgls_device(prob, niter, x0=x0, tol=kwargs.get("tol"), true_residual=kwargs.get("true_residual", False),
                           restart=kwargs.get("restart", True), verbose=kwargs.get("verbose", False))
    out = prob.out(x)
    if kwargs.get("computel2", False) or kwargs.get("return_residuals", False):
        return out, l2.reshape(1, -1).astype(np.float32)
    return out


def _norm(t):
    """FP64 2-norm of a device tensor (FP64 accumulation kernel)."""
    return float(P.sumsq(t).sqrt().item())


def _residual(prob, x):
    return _norm(prob.b - P.ax(x, prob.plan, "Siddon"))


def lsqr_device(prob: Problem, niter, x0=None, verbose=False):
    """LSQR of krylov_subspace_algorithms.py:101-187 (Paige & Saunders): Siddon / matched pair,
    vectors resident on the device, scalar recurrences in FP64 on the host.  The logged
    residual is the explicit |b - A x| of the reference (:174); when it grows, the last step is
    undone and the iteration stops (:175-187)."""
    T = torch()
    plan = prob.plan
    x = prob.zeros_vol() if x0 is None else prob.to_device_vol(x0)
    u = prob.b - P.ax(x, plan, "Siddon")
    beta = _norm(u)
    u.div_(beta)
    phibar = beta
    v = P.atb(u, plan, "matched")
    alpha = _norm(v)
    v.div_(alpha)
    rhobar = alpha
    w = v.clone()
    tmp_p = T.empty_like(u)
    tmp_v = T.empty_like(v)
    l2 = []
    for it in range(niter):
        P.ax(v, plan, "Siddon", out=tmp_p)
        u = tmp_p - alpha * u
        beta = _norm(u)
        u.div_(beta)
        P.atb(u, plan, "matched", out=tmp_v)
        v = tmp_v - beta * v
        alpha = _norm(v)
        v.div_(alpha)
        rho = float(np.hypot(rhobar, beta))
        c, s = rhobar / rho, beta / rho
        theta = s * alpha
        rhobar = -c * alpha
        phi = c * phibar
        phibar = s * phibar
        w_old = w
        x.add_(w_old, alpha=phi / rho)
        w = v - (theta / rho) * w_old
        res = _residual(prob, x)
        if it > 0 and res > l2[-1]:
            x.add_(w_old, alpha=-phi / rho)
            if verbose:
                print("LSQR exited due to divergence at iteration", it)
            break
        l2.append(res)
    return x, np.asarray(l2, dtype=np.float64)


def lsmr_device(prob: Problem, niter, x0=None, lmbda=1.0, verbose=False):
    """LSMR of krylov_subspace_algorithms.py:299-439 (Fong & Saunders) with damping lmbda (the
    reference passes its generic lmbda, default 1).  Same pair, residual log and divergence
    rule as lsqr_device."""
    plan = prob.plan
    x = prob.zeros_vol() if x0 is None else prob.to_device_vol(x0)
    u = prob.b - P.ax(x, plan, "Siddon")
    beta = _norm(u)
    u.div_(beta)
    v = P.atb(u, plan, "matched")
    alpha = _norm(v)
    v.div_(alpha)
    alphabar, zetabar = alpha, alpha * beta
    rho, rhobar, cbar, sbar = 1.0, 1.0, 1.0, 0.0
    h = v.clone()
    hbar = None
    zeta = 0.0
    l2 = []
    for it in range(niter):
        u = P.ax(v, plan, "Siddon") - alpha * u
        beta = _norm(u)
        u.div_(beta)
        v = P.atb(u, plan, "matched") - beta * v
        alpha = _norm(v)
        v.div_(alpha)
        alphahat = float(np.hypot(alphabar, lmbda))
        rhopre = rho
        rho = float(np.hypot(alphahat, beta))
        c, s = alphahat / rho, beta / rho
        theta = s * alpha
        alphabar = c * alpha
        thetabar = sbar * rho
        rhobarpre = rhobar
        rhobar = float(np.hypot(cbar * rho, theta))
        cbar = cbar * rho / rhobar
        sbar = theta / rhobar
        zeta = cbar * zetabar
        zetabar = -sbar * zetabar
        hbar = h.clone() if hbar is None else h - (thetabar * rho / (rhopre * rhobarpre)) * hbar
        step = zeta / (rho * rhobar)
        x.add_(hbar, alpha=step)
        h = v - (theta / rho) * h
        res = _residual(prob, x)
        if it > 0 and res > l2[-1]:
            x.add_(hbar, alpha=-step)
            if verbose:
                print("LSMR exited due to divergence at iteration", it)
            break
        l2.append(res)
    return x, np.asarray(l2, dtype=np.float64)


def _krylov_entry(solver, proj, geo, angles, niter, kwargs, **extra):
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
    x, l2 = solver(prob, niter, x0=x0, verbose=kwargs.get("verbose", False), **extra)
    out = prob.out(x)
    if kwargs.get("computel2", False):
        return out, l2.reshape(1, -1).astype(np.float32)
    return out


def lsqr(proj, geo, angles, niter, **kwargs):
    """Drop-in for tigre.algorithms.lsqr(proj, geo, angles, niter, init=, computel2=, gpuids=, verbose=)."""
    return _krylov_entry(lsqr_device, proj, geo, angles, niter, kwargs)


def lsmr(proj, geo, angles, niter, **kwargs):
    """Drop-in for tigre.algorithms.lsmr(proj, geo, angles, niter, lmbda=, init=, computel2=, gpuids=, verbose=)."""
    return _krylov_entry(lsmr_device, proj, geo, angles, niter, kwargs, lmbda=float(kwargs.get("lmbda", 1.0)))
