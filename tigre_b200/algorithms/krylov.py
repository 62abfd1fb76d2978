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
from ..utilities.Measure_Quality import QualityLog
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
    quality = QualityLog(kwargs.get("Quameasopts"), niter)
    callback = None
    if quality.active:
        quality.before(prob.to_device_vol(x0) if x0 is not None else prob.zeros_vol())

        def callback(it, x, rel):
            quality.after(x, it)
            quality.before(x)
    x, l2, _ = cgls_device(prob, niter, x0=x0, tol=kwargs.get("tol"), true_residual=kwargs.get("true_residual", False),
                           restart=kwargs.get("restart", True), verbose=kwargs.get("verbose", False),
                           callback=callback)
    out = prob.out(x)
    if quality.active:
        return out, quality.errors(l2 if kwargs.get("computel2", False) else None)
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


# ---------------------------------------------------------------------------------------
# Hybrid LSQR, AB-/BA-GMRES, IRN-TV-CGLS (krylov_subspace_algorithms.py:190-697).  Vectors
# stay on the device; the small projected problems (SVD, least squares) are solved on the host
# in FP64.  Divergence rule of those drivers: with restart=True (the default) they stop only
# when the residual grows at the second iteration, otherwise on any growth.  When they stop,
# the reference's run_main_iter returns an iterate that its decorator discards, so its callers
# get the initial image back; here the iterate of the last non-growing iteration is returned.
# ---------------------------------------------------------------------------------------

def _dot(a, b):
    T = torch()
    out = T.zeros((), dtype=T.float64, device=a.device)
    P.dot(a.reshape(-1), b.reshape(-1), out=out)
    return float(out.item())


def _stop(i, l2, restart):
    return i > 0 and l2[i] > l2[i - 1] and (i == 1 or not restart)


def hybrid_lsqr_device(prob: Problem, niter, x0=None, lmbda=1.0, restart=True, verbose=False):
    """hybrid_LSQR (krylov_subspace_algorithms.py:190-296): Golub-Kahan bidiagonalisation with
    Tikhonov regularisation lmbda on the projected problem, solved by the SVD of B_k^T each
    iteration.  The reference's re-orthogonalisation against the older basis vectors
    (j < i-1) is elementwise (v -= V_j * v * V_j); it is kept as written."""
    T = torch()
    plan = prob.plan
    x = prob.zeros_vol() if x0 is None else prob.to_device_vol(x0)
    u = prob.b - P.ax(x, plan, "Siddon")
    normr = _norm(u)
    u = u / normr
    U = [u]
    V = []
    B = np.zeros((niter, niter + 1))
    rhs = np.zeros(niter + 1)
    rhs[0] = normr
    beta = normr
    l2 = []
    best = x
    for i in range(niter):
        v = P.atb(u, plan, "matched")
        if i > 0:
            v = v - beta * V[i - 1]
        for j in range(i - 1):
            v = v - V[j] * v * V[j]
        alpha = _norm(v)
        v = v / alpha
        V.append(v)
        u = P.ax(v, plan, "Siddon") - alpha * u
        for j in range(i - 1):
            u = u - U[j] * u * U[j]
        beta = _norm(u)
        u = u / beta
        U.append(u)
        B[i, i] = alpha
        B[i, i + 1] = beta
        Uk, Sk, Vh = np.linalg.svd(B[:i + 1, :i + 2].T)
        rk = Uk.T @ rhs[:i + 2]
        y = Vh.T @ (Sk * rk[:i + 1] / (Sk ** 2 + lmbda ** 2))
        xi = x.clone()
        for j in range(i + 1):
            xi.add_(V[j], alpha=float(y[j]))
        l2.append(_residual(prob, xi))
        if _stop(i, l2, restart):
            if verbose:
                print("hybrid LSQR exited due to divergence at iteration", i)
            return best, np.asarray(l2[:-1], dtype=np.float64)
        best = xi
    return best, np.asarray(l2, dtype=np.float64)


def _gmres(prob, niter, x0, backprojector, space, restart, verbose):
    """AB-GMRES (space = 'proj', :570-631) and BA-GMRES (space = 'vol', :634-695): Arnoldi with
    modified Gram-Schmidt on A B (AB) or B A (BA), B the matched or FDK backprojector, and the
    small least-squares problem min |H_k^T y - |r| e1| on the host.  AB keeps B w_i of every
    basis vector, so the iterate x + sum_i y_i B w_i needs no extra backprojections."""
    plan = prob.plan
    T = torch()
    if backprojector == "matched":
        back = lambda t: P.atb(t.contiguous(), plan, "matched")  # noqa: E731
    elif backprojector == "FDK":
        from .single_pass import fdk_device
        back = lambda t: fdk_device(prob, proj=t.contiguous())  # noqa: E731
    else:
        raise ValueError("backprojector must be 'matched' or 'FDK'")
    x = prob.zeros_vol() if x0 is None else prob.to_device_vol(x0)
    r = prob.b - P.ax(x, plan, "Siddon")
    if space == "vol":
        r = back(r)
    rnorm = _norm(r)
    W = [r / rnorm]
    Z = []            # AB: B w_i (volume); BA: w_i itself
    H = np.zeros((niter, niter + 1))
    l2 = []
    best = x
    for k in range(niter):
        if space == "proj":
            z = back(W[k])
            Z.append(z)
            q = P.ax(z, plan, "Siddon")
        else:
            Z.append(W[k])
            q = back(P.ax(W[k], plan, "Siddon"))
        for i in range(k + 1):
            H[k, i] = _dot(q, W[i])
            q = q - float(H[k, i]) * W[i]
        H[k, k + 1] = _norm(q)
        W.append(q / float(H[k, k + 1]))
        e1 = np.zeros(k + 2)
        e1[0] = rnorm
        y = np.linalg.lstsq(H[:k + 1, :k + 2].T, e1, rcond=None)[0]
        xi = x.clone()
        for i in range(k + 1):
            xi.add_(Z[i], alpha=float(np.float32(y[i])))
        l2.append(_residual(prob, xi))
        if _stop(k, l2, restart):
            if verbose:
                print(("AB" if space == "proj" else "BA") + "-GMRES exited due to divergence at iteration", k)
            return best, np.asarray(l2[:-1], dtype=np.float64)
        best = xi
    del T
    return best, np.asarray(l2, dtype=np.float64)


def _diff_stack(img):
    """The differences of IRN_TV_CGLS.Lx (:473-480) along each axis of (nZ, nY, nX): a copy of
    the image whose first n-2 entries along the axis become img[i] - img[i+1] (the last two keep
    the image values, as the reference's slices do)."""
    out = []
    for ax in range(3):
        d = img.clone()
        n = img.shape[ax]
        if n > 2:
            d.narrow(ax, 0, n - 2).copy_(img.narrow(ax, 0, n - 2) - img.narrow(ax, 1, n - 2))
        out.append(d)
    return out


def _irn_weights(x):
    d = _diff_stack(x)
    return (d[0] ** 2 + d[1] ** 2 + d[2] ** 2 + 1e-6) ** (-0.25)


def _Lx(Wt, img):
    T = torch()
    return T.stack([Wt * d for d in _diff_stack(img)], dim=0)


def _Ltx(Wt, img3):
    """IRN_TV_CGLS.Ltx (:482-500): per axis W*g with entries 1..n-3 replaced by the backward
    difference, entry n-1 by -(W*g)[n-2]; entries 0 and n-2 keep W*g."""
    acc = None
    for ax in range(3):
        wg = Wt * img3[ax]
        o = wg.clone()
        n = wg.shape[ax]
        if n > 3:
            o.narrow(ax, 1, n - 3).copy_(wg.narrow(ax, 1, n - 3) - wg.narrow(ax, 0, n - 3))
        if n >= 2:
            o.narrow(ax, n - 1, 1).copy_(-wg.narrow(ax, n - 2, 1))
        acc = o if acc is None else acc + o
    return acc


def irn_tv_cgls_device(prob: Problem, niter, x0=None, lmbda=1.0, niter_outer=4, verbose=False):
    """IRN_TV_CGLS (:441-567): niter_outer reweightings, each niter CGLS steps on
    [A; sqrt(lmbda) W D].  As the reference, every outer pass restarts from the iterate
    before the last inner update of the previous pass (its res0 bookkeeping, :526-536)."""
    plan = prob.plan
    sl = float(np.sqrt(lmbda))
    x = prob.zeros_vol() if x0 is None else prob.to_device_vol(x0)
    x0_ = x
    l2 = []
    for outer in range(niter_outer):
        Wt = _irn_weights(x)
        x = x0_
        r1 = prob.b - P.ax(x, plan, "Siddon")
        r2 = -_Lx(Wt, x) * sl
        p = P.atb(r1.contiguous(), plan, "matched") + sl * _Ltx(Wt, r2)
        gamma = _norm(p) ** 2
        for i in range(niter):
            x0_ = x
            q1 = P.ax(p.contiguous(), plan, "Siddon")
            q2 = _Lx(Wt, p) * sl
            alpha = gamma / (_norm(q1) ** 2 + _norm(q2) ** 2)
            x = x + alpha * p
            l2.append(_residual(prob, x))
            r1 = r1 - alpha * q1
            r2 = r2 - alpha * q2
            s = P.atb(r1.contiguous(), plan, "matched") + sl * _Ltx(Wt, r2)
            gamma1 = _norm(s) ** 2
            beta = gamma1 / gamma
            gamma = gamma1
            p = s + beta * p
        if verbose:
            print("IRN-TV-CGLS outer iteration", outer)
    return x, np.asarray(l2, dtype=np.float64)


def hybrid_lsqr(proj, geo, angles, niter, **kwargs):
    """Drop-in for tigre.algorithms.hybrid_lsqr(proj, geo, angles, niter, lmbda=1, init=, computel2=, restart=)."""
    return _krylov_entry(hybrid_lsqr_device, proj, geo, angles, niter, kwargs, lmbda=float(kwargs.get("lmbda", 1.0)),
                         restart=kwargs.get("restart", True))


def ab_gmres(proj, geo, angles, niter, **kwargs):
    """Drop-in for tigre.algorithms.ab_gmres(..., backprojector="matched" | "FDK")."""
    return _krylov_entry(lambda prob, n, x0=None, verbose=False, **kw: _gmres(prob, n, x0, kw["bp"], "proj",
                                                                               kw["restart"], verbose),
                         proj, geo, angles, niter, kwargs, bp=kwargs.get("backprojector", "matched"),
                         restart=kwargs.get("restart", True))


def ba_gmres(proj, geo, angles, niter, **kwargs):
    """Drop-in for tigre.algorithms.ba_gmres(..., backprojector="matched" | "FDK")."""
    return _krylov_entry(lambda prob, n, x0=None, verbose=False, **kw: _gmres(prob, n, x0, kw["bp"], "vol",
                                                                               kw["restart"], verbose),
                         proj, geo, angles, niter, kwargs, bp=kwargs.get("backprojector", "matched"),
                         restart=kwargs.get("restart", True))


def irn_tv_cgls(proj, geo, angles, niter, **kwargs):
    """Drop-in for tigre.algorithms.irn_tv_cgls(..., lmbda=1, niter_outer=4)."""
    return _krylov_entry(irn_tv_cgls_device, proj, geo, angles, niter, kwargs, lmbda=float(kwargs.get("lmbda", 1.0)),
                         niter_outer=int(kwargs.get("niter_outer", 4)))


def _sym_ortho(a, b):
    """Stable Givens rotation (c, s, r) with r = hypot(a, b) (Paige & Saunders' LSQR)."""
    if b == 0.0:
        return float(np.sign(a)), 0.0, abs(a)
    if a == 0.0:
        return 0.0, float(np.sign(b)), abs(b)
    if abs(b) > abs(a):
        tau = a / b
        s_ = float(np.sign(b)) / np.sqrt(1.0 + tau * tau)
        return s_ * tau, s_, b / s_
    tau = b / a
    c = float(np.sign(a)) / np.sqrt(1.0 + tau * tau)
    return c, c * tau, a / c


def _lsqr_op(A, At, b, x_like, iter_lim, atol=1e-6, btol=1e-6, conlim=1e8):
    """LSQR (Paige & Saunders 1982) for min |A x - b| with device vectors, no damping, and the
    stopping tests of scipy.sparse.linalg.lsqr, which the reference's hybrid_fLSQR_TV calls with
    iter_lim=50 (:777-780).  A maps x_like-shaped tensors to b-shaped ones."""
    T = torch()
    x = T.zeros_like(x_like)
    u = b.clone()
    bnorm = _norm(u)
    beta = bnorm
    if beta > 0:
        u = u / beta
        v = At(u)
        alpha = _norm(v)
    else:
        return x
    if alpha > 0:
        v = v / alpha
    w = v.clone()
    rhobar, phibar = alpha, beta
    anorm = acond = ddnorm = res2 = xxnorm = z = 0.0
    cs2, sn2 = -1.0, 0.0
    if alpha * beta == 0:
        return x
    ctol = 1.0 / conlim
    eps = np.finfo(np.float64).eps
    for itn in range(1, iter_lim + 1):
        u = A(v) - alpha * u
        beta = _norm(u)
        if beta > 0:
            u = u / beta
            anorm = np.sqrt(anorm ** 2 + alpha ** 2 + beta ** 2)
            v = At(u) - beta * v
            alpha = _norm(v)
            if alpha > 0:
                v = v / alpha
        cs, sn, rho = _sym_ortho(rhobar, beta)
        theta = sn * alpha
        rhobar = -cs * alpha
        phi = cs * phibar
        phibar = sn * phibar
        tau = sn * phi
        ddnorm += (_norm(w) / rho) ** 2
        x = x + (phi / rho) * w
        w = v + (-theta / rho) * w
        delta = sn2 * rho
        gambar = -cs2 * rho
        rhs = phi - delta * z
        zbar = rhs / gambar
        xnorm = np.sqrt(xxnorm + zbar ** 2)
        gamma = np.sqrt(gambar ** 2 + theta ** 2)
        cs2, sn2 = gambar / gamma, theta / gamma
        z = rhs / gamma
        xxnorm += z ** 2
        acond = anorm * np.sqrt(ddnorm)
        rnorm = np.sqrt(phibar ** 2 + res2)
        arnorm = alpha * abs(tau)
        test1 = rnorm / bnorm
        test2 = arnorm / (anorm * rnorm + eps)
        test3 = 1.0 / (acond + eps)
        t1 = test1 / (1.0 + anorm * xnorm / bnorm)
        rtol = btol + atol * anorm * xnorm / bnorm
        if (itn >= iter_lim or 1 + test3 <= 1 or 1 + test2 <= 1 or 1 + t1 <= 1 or test3 <= ctol or test2 <= atol
                or test1 <= rtol):
            break
    return x


def hybrid_flsqr_tv_device(prob: Problem, niter, x0=None, lmbda=1.0, restart=True, verbose=False):
    """hybrid_fLSQR_TV (krylov_subspace_algorithms.py:698-858): flexible Golub-Kahan with the
    TV-weighted preconditioner applied by two inner LSQR solves on the difference operator
    (50 iterations each), the mean-value component split off through k_aux, and the projected
    problem [M_k^T; lmbda R_k] y = [|r| e1; 0] with R_k^T R_k the Gram matrix of W D Z_j.
    The reference's run_main_iter returns its iterate without storing it, so its decorator
    hands back the initial image; here the iterate is returned."""
    T = torch()
    plan = prob.plan
    x = prob.zeros_vol() if x0 is None else prob.to_device_vol(x0)
    nvox = float(np.prod(prob.vol_shape))
    u = prob.b - P.ax(x, plan, "Siddon")
    ones = T.ones_like(x) / np.sqrt(nvox)
    k_aux = P.ax(ones, plan, "Siddon")
    kn2 = _norm(k_aux) ** 2
    xA0 = T.full_like(x, _dot(k_aux, u) / (np.sqrt(nvox) * kn2))
    k_aux = P.atb(k_aux, plan, "matched") / (np.sqrt(nvox) * kn2)
    u = u - P.ax(xA0, plan, "Siddon")
    normr = _norm(u)
    u = u / normr
    U, V, Z, LZ = [u], [], [], []
    M = np.zeros((niter, niter + 1))
    rhs = np.zeros(niter + 1)
    rhs[0] = normr
    Wt = T.ones_like(x) if float(x.max().item()) == 0.0 else _irn_weights(x)
    Lx = lambda t: _Lx(Wt, t.reshape(x.shape))  # noqa: E731
    Ltx = lambda t: _Ltx(Wt, t.reshape((3,) + tuple(x.shape)))  # noqa: E731
    G = np.zeros((niter, niter))
    l2 = []
    best = x + xA0
    for i in range(niter):
        v = P.atb(u.contiguous(), plan, "matched")
        for j in range(i):
            v = v - _dot(V[j], v) * V[j]
        v = v / _norm(v)
        zt = v - k_aux * float(v.sum(dtype=T.float64).item())
        aux = _lsqr_op(Ltx, Lx, zt.contiguous(), T.zeros((3,) + tuple(x.shape), device=x.device), 50)
        zt = _lsqr_op(Lx, Ltx, aux.contiguous(), x, 50)
        zt = zt - _dot(k_aux, zt.contiguous())
        V.append(v)
        Z.append(zt.contiguous())
        u = P.ax(Z[i], plan, "Siddon")
        for j in range(i + 1):
            M[i, j] = _dot(U[j], u)
            u = u - M[i, j] * U[j]
        M[i, i + 1] = _norm(u)
        u = u / M[i, i + 1]
        U.append(u)
        LZ.append(Lx(Z[i]).contiguous())
        for j in range(i + 1):
            G[i, j] = G[j, i] = _dot(LZ[i], LZ[j])
        ev, evec = np.linalg.eigh(G[:i + 1, :i + 1])
        R = np.sqrt(np.clip(ev, 0.0, None))[:, None] * evec.T          # R^T R = G
        MZ = np.concatenate([M[:i + 1, :i + 2].T, lmbda * R])
        rz = np.concatenate([rhs[:i + 2], np.zeros(i + 1)])
        y = np.linalg.lstsq(MZ, rz, rcond=None)[0]
        xi = x + xA0
        for j in range(i + 1):
            xi.add_(Z[j], alpha=float(y[j]))
        l2.append(_residual(prob, xi))
        if _stop(i, l2, restart):
            if verbose:
                print("hybrid fLSQR-TV exited due to divergence at iteration", i)
            return best, np.asarray(l2[:-1], dtype=np.float64)
        best = xi
    return best, np.asarray(l2, dtype=np.float64)


def hybrid_flsqr_tv(proj, geo, angles, niter, **kwargs):
    """Drop-in for tigre.algorithms.hybrid_flsqr_tv(proj, geo, angles, niter, lmbda=1, init=, computel2=)."""
    return _krylov_entry(hybrid_flsqr_tv_device, proj, geo, angles, niter, kwargs,
                         lmbda=float(kwargs.get("lmbda", 1.0)), restart=kwargs.get("restart", True))
