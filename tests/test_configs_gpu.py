"""The plain-method configurations, at their own sizes, through the product path, against the
FP64 oracle (bar 1e-5 relative unless stated).

C1  64^3 @ 1 mm, 128 x 128 detector @ 0.8 mm, DSO 1000 / DSD 1536 mm, 100 views over 2 pi:
    10 CGLS iterations (Siddon Ax, matched Atb) against the oracle CGLS.
C2  256^3 @ 1 mm, 512 x 512 detector @ 0.8 mm: interpolated Ax of 360 views over 2 pi (all views
    on the GPU; views and rows compared with the oracle); FDK with the Ram-Lak filter and Parker
    weights on the short scan of 360 views over [0, pi + 2 delta], delta = atan(0.5 * 409.6 / 1536)
    (end angle included), of interpolated projections with Poisson noise at I0 = 1e5 (slices
    compared with the oracle FDK of the same noisy projections).
C4  batch of 8 128^3 @ 1 mm phantoms, 256 x 256 detector @ 0.8 mm, 180 views: the autograd
    operator's backward against the matched backprojector, the adjoint dot test, and central
    differences at h = 1e-3 of |Ax - b|^2 + 1e-3 TV(x).
"""
import warnings

import numpy as np
import pytest

from tests import geometries as G
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _cone(n, vox_mm, nd, det_mm):
    from tigre_b200.utilities.geometry import cone_geometry
    return cone_geometry((n, n, n), (n * vox_mm,) * 3, (nd, nd), (det_mm, det_mm), DSO=1000.0, DSD=1536.0)


# ------------------------------------------------------------------------------------------ C1 --
def test_c1_cgls_ten_iterations_matches_oracle():
    import tigre_b200 as tigre
    geo = _cone(64, 1.0, 128, 0.8)
    ang = np.linspace(0, 2 * np.pi, 100, endpoint=False).astype(np.float32)
    img = G.phantom((64, 64, 64), seed=0)
    proj = O.ax(img, geo, ang, "Siddon")
    x, res = tigre.algorithms.cgls(proj, geo, ang, 10, computel2=True)
    xr, resr = O.cgls(proj, geo, ang, 10)
    assert len(resr) == 10
    mx, l2 = G.rel_err(x, xr)
    print("C1 CGLS 10 iterations vs FP64 oracle: max %.2e, L2 %.2e" % (mx, l2))
    assert l2 <= 1e-4 and mx <= 1e-3, (mx, l2)
    np.testing.assert_allclose(np.asarray(res).ravel()[:10], resr, rtol=1e-4)


# ------------------------------------------------------------------------------------------ C2 --
C2_DELTA = float(np.arctan(0.5 * 409.6 / 1536.0))


def _c2():
    geo = _cone(256, 1.0, 512, 0.8)
    img = G.phantom((256, 256, 256), seed=0)
    return geo, img


def test_c2_interpolated_projection_matches_oracle():
    import torch
    import tigre_b200 as tigre
    geo, img = _c2()
    ang = np.linspace(0, 2 * np.pi, 360, endpoint=False).astype(np.float32)
    got = tigre.Ax(torch.from_numpy(img).cuda(), geo, ang, "interpolated").cpu().numpy()
    assert got.shape == (360, 512, 512)
    for a0 in (0, 45, 181, 302):
        for r0, r1 in ((0, 64), (224, 288), (448, 512)):
            ref = O.ax(img, geo, ang, "interpolated", angle_range=(a0, a0 + 2), row_range=(r0, r1))
            mx, l2 = G.rel_err(got[a0:a0 + 2, r0:r1], ref)
            assert mx <= TOL and l2 <= TOL, (a0, r0, mx, l2)


def test_c2_short_scan_parker_fdk_with_poisson_noise_matches_oracle():
    import torch
    import tigre_b200 as tigre
    from tigre_b200.utilities import CTnoise
    geo, img = _c2()
    ang = np.linspace(0, np.pi + 2 * C2_DELTA, 360).astype(np.float32)
    clean = tigre.Ax(torch.from_numpy(img).cuda(), geo, ang, "interpolated")
    noisy = CTnoise.add(clean, Poisson=1e5, Gaussian=np.array([0.0, 0.0]))
    noisy_np = noisy.cpu().numpy()
    assert np.isfinite(noisy_np).all()
    # the noise has the size Poisson statistics give it: var(p) ~ max(p)^2 / (I0 exp(-p / max p))
    clean_np = clean.cpu().numpy()
    pmax = float(clean_np.max())
    sel = clean_np > 0.05 * pmax
    z = (noisy_np - clean_np)[sel] / (pmax / np.sqrt(1e5 * np.exp(-clean_np[sel] / pmax)))
    assert abs(float(np.std(z)) - 1.0) < 0.05 and abs(float(np.mean(z))) < 0.05, (np.std(z), np.mean(z))
    with warnings.catch_warnings():
        # a proper short scan: neither Parker warning nor a division by zero may occur
        warnings.simplefilter("error", UserWarning)
        warnings.simplefilter("error", RuntimeWarning)
        rec = tigre.algorithms.fdk(noisy_np, geo, ang, parker=True)
        assert rec.shape == (256, 256, 256)
        for z0 in (40, 127, 230):
            ref = O.fdk(noisy_np, geo, ang, parker=True, z_range=(z0, z0 + 2))
            mx, l2 = G.rel_err(rec[z0:z0 + 2], ref)
            assert mx <= 2e-5 and l2 <= TOL, (z0, mx, l2)
    # Parker weighting is what makes the short scan reconstruct: the central slab is closer to
    # the phantom with it than without (plain FDK double-counts the overlap region)
    plain = tigre.algorithms.fdk(noisy_np, geo, ang)
    c = slice(96, 160)
    e_park = np.linalg.norm(rec[c] - img[c])
    e_plain = np.linalg.norm(plain[c] - img[c])
    print("C2 short scan, central slab error vs phantom: Parker FDK %.4g, plain FDK %.4g" % (e_park, e_plain))
    assert e_park < e_plain, (e_park, e_plain)


# ------------------------------------------------------------------------------------------ C4 --
def _c4():
    import torch
    geo = _cone(128, 1.0, 256, 0.8)
    ang = np.linspace(0, 2 * np.pi, 180, endpoint=False).astype(np.float32)
    vols = np.stack([G.phantom((128, 128, 128), seed=s) for s in range(8)])
    return geo, ang, torch.from_numpy(vols).cuda()


def test_c4_batched_autograd_adjoint():
    """Backward of the batched operator = matched backprojection of each element; dot-test gap
    of the matched pair below 2 %."""
    import torch
    from tigre_b200 import autograd as AG, projectors as P
    geo, ang, x = _c4()
    A = AG.A(geo, ang)
    xg = x.clone().requires_grad_(True)
    y = torch.rand((8, 180, 256, 256), device="cuda", generator=torch.Generator("cuda").manual_seed(1))
    Ax = A(xg)
    assert Ax.shape == (8, 180, 256, 256)
    (Ax * y).sum().backward()
    for i in (0, 5):
        torch.testing.assert_close(xg.grad[i], P.atb(y[i].contiguous(), A.plan, "matched"), rtol=0, atol=0)
    lhs = float((Ax.detach().double() * y.double()).sum())
    rhs = float((x.double() * xg.grad.double()).sum())
    gap = abs(lhs - rhs) / abs(lhs)
    print("C4 adjoint dot test gap (Siddon vs matched): %.3e" % gap)
    assert gap < 0.02, gap


def test_c4_batched_loss_central_differences():
    """loss = |Ax - b|^2 + 1e-3 TV(x) over the batch, central differences at h = 1e-3 along
    smooth directions (a Gaussian blob in every batch element).  The backward of Ax is the
    matched backprojector, the reference's adjoint of Siddon up to its weights' small mismatch
    (measured 1.8e-3 along these directions), so the bar is 5e-3 relative: the residual
    Ax0 - b is kept systematic (x0 = 1.05 x + noise)
    so that <r, A d> is not a near-cancelling sum of signed noise, which would magnify that
    mismatch.  The TV term's backward is exact: checked along random directions at 2e-3."""
    import torch
    from tigre_b200 import autograd as AG, projectors as P
    geo, ang, x = _c4()
    A = AG.A(geo, ang)
    g = torch.Generator("cuda").manual_seed(2)
    b = A(x).double()
    x0 = 1.05 * x + 0.02 * torch.randn(x.shape, device="cuda", generator=g)
    h = 1e-3

    def data(v):
        r = A(v).double() - b
        return (r * r).sum()

    def loss(v):
        return data(v) + 1e-3 * AG.tv(v).double()

    def grad(f):
        v = x0.clone().requires_grad_(True)
        f(v).backward()
        return v.grad.double()

    def fd(f, d):
        return (f(x0 + h * d) - f(x0 - h * d)).item() / (2 * h)

    ax = torch.arange(128, device="cuda", dtype=torch.float32)
    zz, yy, xx = torch.meshgrid(ax, ax, ax, indexing="ij")
    rng = np.random.default_rng(3)
    g_data, g_all = grad(data), grad(loss)
    for _ in range(3):
        d = torch.zeros_like(x0)
        for i in range(8):
            c = rng.uniform(40, 88, 3)
            d[i] = torch.exp(-((zz - c[0]) ** 2 + (yy - c[1]) ** 2 + (xx - c[2]) ** 2) / (2 * 8.0 ** 2))
        e_data = abs(fd(data, d) - float((g_data * d).sum())) / abs(fd(data, d))
        e_all = abs(fd(loss, d) - float((g_all * d).sum())) / abs(fd(loss, d))
        print("C4 central differences: data %.3e, data + TV %.3e" % (e_data, e_all))
        assert e_data < 5e-3 and e_all < 5e-3, (e_data, e_all)
    # TV alone along random directions (FP64 sums; shifted away from the kink at 0 as in the
    # small-size check)
    x1 = x0 + 4.0
    g1 = torch.stack([P.tv_gradient(x1[i].contiguous()).double() for i in range(8)])
    for seed in range(2):
        d = torch.randn(x1.shape, device="cuda", generator=torch.Generator("cuda").manual_seed(10 + seed))
        tv = lambda v: sum(P.tv_value(v[i].contiguous()).item() for i in range(8))  # noqa: E731
        ref = (tv(x1 + 1e-4 * d) - tv(x1 - 1e-4 * d)) / 2e-4
        assert abs(ref - float((g1 * d).sum())) <= 2e-3 * abs(ref), (seed, ref)
