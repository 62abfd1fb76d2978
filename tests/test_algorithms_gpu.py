"""Algorithm drivers and autograd on the GPU, checked against oracle restatements."""
import numpy as np
import pytest

from tests import geometries as G
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _case(n=32, views=24, seed=3):
    from tigre_b200.utilities.geometry import cone_geometry
    geo = cone_geometry((n, n, n), (float(n),) * 3, (48, 64), (0.8, 0.8))
    ang = G.angles(views)
    img = G.phantom((n, n, n), seed=seed)
    return geo, ang, img


def test_cgls_matches_oracle_cgls():
    import tigre_b200 as tigre
    geo, ang, img = _case()
    proj = O.ax(img, geo, ang, "Siddon")
    x, l2 = tigre.algorithms.cgls(proj, geo, ang, 6, computel2=True)
    xr, resr = O.cgls(proj, geo, ang, 6)
    mx, l2e = G.rel_err(x, xr)
    assert l2e <= 1e-4, (mx, l2e)
    np.testing.assert_allclose(l2.ravel()[:len(resr)], resr, rtol=1e-4)
    assert np.all(np.diff(l2.ravel()) < 0)


def test_cgls_tol_stops_early_and_device_input():
    import torch
    import tigre_b200 as tigre
    geo, ang, img = _case()
    proj = torch.from_numpy(O.ax(img, geo, ang, "Siddon")).cuda()
    x, l2 = tigre.algorithms.cgls(proj, geo, ang, 200, tol=1e-2, computel2=True)
    assert x.is_cuda
    b = float(torch.linalg.vector_norm(proj.double()))
    assert l2.ravel()[-1] <= 1e-2 * b and l2.size < 200


@pytest.mark.parametrize("filt", [None, "hann"])
def test_fdk_matches_oracle(filt):
    import tigre_b200 as tigre
    geo, ang, img = _case(views=40)
    proj = O.ax(img, geo, ang, "Siddon")
    got = tigre.algorithms.fdk(proj, geo, ang, filter=filt)
    ref = O.fdk(proj, geo, ang, filt)
    mx, l2 = G.rel_err(got, ref)
    assert mx <= 2e-5 and l2 <= 1e-5, (mx, l2)


def test_parker_short_scan_fdk_improves_on_plain():
    import tigre_b200 as tigre
    from tigre_b200.utilities.geometry import cone_geometry
    geo = cone_geometry((48, 48, 48), (48.0,) * 3, (64, 96), (0.8, 0.8))
    delta = np.arctan(0.5 * 96 * 0.8 / 1536.0)
    ang = np.linspace(0, np.pi + 2 * delta, 90, endpoint=False).astype(np.float32)
    img = G.phantom((48, 48, 48), seed=5)
    proj = O.ax(img, geo, ang, "Siddon")
    plain = tigre.algorithms.fdk(proj, geo, ang)
    park = tigre.algorithms.fdk(proj, geo, ang, parker=True)
    e_plain = np.linalg.norm(plain - img)
    e_park = np.linalg.norm(park - img)
    assert np.isfinite(e_park) and e_park < e_plain


def test_ossart_reduces_residual_and_matches_host_update():
    import tigre_b200 as tigre
    geo, ang, img = _case(views=30)
    proj = O.ax(img, geo, ang, "Siddon")
    x, l2 = tigre.algorithms.ossart(proj, geo, ang, 3, blocksize=10, computel2=True)
    assert np.all(np.diff(l2.ravel()) < 0)
    assert np.linalg.norm(x - img) < np.linalg.norm(img)


def test_ossart_bf16_storage_close_to_fp32():
    import torch
    import tigre_b200 as tigre
    geo, ang, img = _case(views=30)
    proj = O.ax(img, geo, ang, "Siddon")
    x32 = tigre.algorithms.ossart(proj, geo, ang, 3, blocksize=10)
    x16 = tigre.algorithms.ossart(proj, geo, ang, 3, blocksize=10, storage=torch.bfloat16)
    rel = np.linalg.norm(x16 - x32) / np.linalg.norm(x32)
    assert rel < 2e-2, rel


def test_asd_pocs_runs_and_reconstructs():
    import tigre_b200 as tigre
    geo, ang, img = _case(views=20)
    proj = O.ax(img, geo, ang, "Siddon")
    x = tigre.algorithms.asd_pocs(proj, geo, ang, 3, tviter=5)
    assert np.linalg.norm(x - img) < 0.8 * np.linalg.norm(img)


def test_autograd_backward_is_matched_adjoint():
    import torch
    from tigre_b200 import autograd as AG, projectors as P
    geo, ang, img = _case()
    A = AG.A(geo, ang)
    x = torch.from_numpy(img).cuda().requires_grad_(True)
    y = torch.rand((24, 48, 64), device="cuda")
    (A(x) * y).sum().backward()
    ref = P.atb(y, A.plan, "matched")
    torch.testing.assert_close(x.grad, ref, rtol=0, atol=0)


def test_autograd_loss_finite_differences():
    """loss = |Ax - b|^2 + 1e-3 TV(x): autograd vs central differences (h = 1e-3).
    The backward of Ax is the matched backprojector, the reference's approximate
    adjoint of Siddon, so agreement is within its adjoint gap (a few %)."""
    import torch
    from tigre_b200 import autograd as AG
    geo, ang, img = _case(n=24, views=18)
    rng = np.random.default_rng(0)
    A = AG.A(geo, ang)
    b = torch.from_numpy(O.ax(img, geo, ang, "Siddon")).cuda().double()
    # noise >> h keeps every |grad f| term of the TV away from its kink during the differences
    x0 = torch.from_numpy((img + rng.normal(0, 5e-2, img.shape)).astype(np.float32)).cuda()

    def loss(x):
        r = A(x).double() - b
        return (r * r).sum() + 1e-3 * AG.tv(x).double()

    x = x0.clone().requires_grad_(True)
    loss(x).backward()
    g = x.grad.double()
    h = 1e-3
    errs = []
    for idx in [(12, 12, 12), (8, 15, 10), (16, 6, 9)]:
        xp = x0.clone(); xp[idx] += h
        xm = x0.clone(); xm[idx] -= h
        fd = (loss(xp) - loss(xm)).item() / (2 * h)
        errs.append(abs(fd - g[idx].item()) / max(abs(fd), 1e-12))
    assert max(errs) < 0.05, errs


def test_autograd_batch_dimension():
    import torch
    from tigre_b200 import autograd as AG, projectors as P
    geo, ang, img = _case()
    A = AG.A(geo, ang)
    xb = torch.stack([torch.from_numpy(img), torch.from_numpy(img[::-1].copy())]).cuda()
    yb = A(xb)
    assert yb.shape == (2, 24, 48, 64)
    torch.testing.assert_close(yb[1], P.ax(xb[1].contiguous(), A.plan, "Siddon"))
