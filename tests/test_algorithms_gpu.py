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


@pytest.mark.parametrize("q", [1.0, 0.5])
def test_parker_short_scan_fdk_matches_oracle(q):
    """Short scan over [0, pi + 2 delta] (delta from the detector's outer edge, end angle
    included) on a non-square detector: Parker-weighted FDK against the oracle's FP64 Parker
    FDK, and closer to the phantom than unweighted FDK."""
    import warnings
    import tigre_b200 as tigre
    from tigre_b200.utilities.geometry import cone_geometry
    geo = cone_geometry((48, 48, 48), (48.0,) * 3, (64, 96), (0.8, 0.8))
    delta = np.arctan(0.5 * 96 * 0.8 / 1536.0)
    ang = np.linspace(0, np.pi + 2 * delta, 91).astype(np.float32)
    img = G.phantom((48, 48, 48), seed=5)
    proj = O.ax(img, geo, ang, "Siddon")
    with warnings.catch_warnings():
        warnings.simplefilter("error", UserWarning)
        warnings.simplefilter("error", RuntimeWarning)
        park = tigre.algorithms.fdk(proj, geo, ang, parker=q)
    mx, l2 = G.rel_err(park, O.fdk(proj, geo, ang, parker=q))
    assert mx <= 2e-5 and l2 <= 1e-5, (mx, l2)
    plain = tigre.algorithms.fdk(proj, geo, ang)
    assert np.linalg.norm(park - img) < np.linalg.norm(plain - img)


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


def _noisy_case():
    """Projections with seeded Gaussian noise: the TV gradient d / (|d| + 1e-8) is ill-conditioned
    on piecewise-constant images (differences at the FP32 rounding level flip it between 0 and
    +-1), so the regulariser checks run on a noisy reconstruction, as a measured one is."""
    geo, ang, img = _case(views=20)
    proj = O.ax(img, geo, ang, "Siddon")
    rng = np.random.default_rng(41)
    return geo, ang, (proj + rng.normal(0, 2e-3, proj.shape)).astype(np.float32)


@pytest.mark.parametrize("name", ["asd_pocs", "awasd_pocs", "piccs", "os_asd_pocs", "os_awasd_pocs", "os_piccs"])
def test_pocs_family_first_iteration_matches_oracle_regulariser(name):
    """One outer iteration from zero: the (OS-)SART sweep, then tviter steps of the family's
    regulariser with dtvg = alpha |x_sart| (pocs_algorithms.py:140-150), checked against the
    oracle's pocs_tv / aw_pocs_tv / piccs_tv applied to the same sweep."""
    import tigre_b200 as tigre
    from tests import golden_cases as GC
    geo, ang, proj = _noisy_case()
    os_ = name.startswith("os_")
    sweep = (tigre.algorithms.ossart(proj, geo, ang, 1, blocksize=5) if os_ else
             tigre.algorithms.sart(proj, geo, ang, 1))
    # 3 TV steps: over more steps a difference driven to ~0 can take either sign in FP32 and
    # FP64 (the gradient d / (|d| + eps) is discontinuous there), which moves single voxels by
    # up to a step; the wiring itself is exact (asd_pocs and minTV of its sweep agree bitwise)
    kw = dict(tviter=3, alpha=0.002, maxl2err=1.0)
    if os_:
        kw["blocksize"] = 5
    prior = GC.piccs_prior(sweep)
    dtvg = 0.002 * float(np.linalg.norm(sweep.astype(np.float64)))
    if name.endswith("awasd_pocs"):
        got = getattr(tigre.algorithms, name)(proj, geo, ang, 1, delta=0.01, **kw)
        ref = O.aw_pocs_tv(sweep, dtvg, 3, 0.01)
    elif name.endswith("piccs"):
        got = getattr(tigre.algorithms, name)(proj, geo, ang, 1, prior=prior, prior_ratio=0.3, **kw)
        ref = O.piccs_tv(sweep, prior, dtvg, 0.3, 3)
    else:
        got = getattr(tigre.algorithms, name)(proj, geo, ang, 1, **kw)
        ref = O.pocs_tv(sweep, dtvg, 3)
        dev = tigre.minTV(sweep, dtvg, 3)
        mx, l2 = G.rel_err(got, dev)
        assert mx <= 1e-6 and l2 <= 1e-7, (name, "wiring", mx, l2)
    mx, l2 = G.rel_err(got, ref)
    assert mx <= 1e-5 and l2 <= 1e-6, (name, mx, l2)


@pytest.mark.parametrize("name", ["pcsd", "aw_pcsd", "os_pcsd", "os_aw_pcsd"])
def test_pcsd_family_first_iteration_matches_oracle_regulariser(name):
    """PCSD with niter=0 runs exactly one iteration (stop rule n_iter > niter,
    pocs_algorithms.py:553): the sweep (|b|^2 > maxl2err), then the regulariser with dtvg = 1.
    The projections are scaled by 1000 so that a unit TV step is small against the image."""
    import tigre_b200 as tigre
    geo, ang, proj = _noisy_case()
    proj = proj * np.float32(1000.0)
    os_ = name.startswith("os_")
    sweep = (tigre.algorithms.ossart(proj, geo, ang, 1, blocksize=5) if os_ else
             tigre.algorithms.sart(proj, geo, ang, 1))
    kw = dict(tviter=2, maxl2err=1e-9)
    if os_:
        kw["blocksize"] = 5
    if "aw" in name:
        got = getattr(tigre.algorithms, name)(proj, geo, ang, 0, delta=10.0, **kw)
        ref = O.aw_pocs_tv(sweep, 1.0, 2, 10.0)
    else:
        got = getattr(tigre.algorithms, name)(proj, geo, ang, 0, **kw)
        ref = O.pocs_tv(sweep, 1.0, 2)
    mx, l2 = G.rel_err(got, ref)
    assert mx <= 1e-4 and l2 <= 1e-5, (name, mx, l2)


def test_pocs_family_runs_and_reconstructs():
    import tigre_b200 as tigre
    geo, ang, img = _case(views=20)
    proj = O.ax(img, geo, ang, "Siddon")
    prior = (0.9 * img).astype(np.float32)
    for name, kw in [("awasd_pocs", {}), ("os_awasd_pocs", {"blocksize": 5}), ("piccs", {"prior": prior}),
                     ("os_piccs", {"prior": prior, "blocksize": 5}), ("pcsd", {}), ("aw_pcsd", {"delta": 5.0})]:
        # PCSD's first TV step is 1 in absolute units (pocs_algorithms.py:527): scale the data so
        # that the image norm is large against it, as for attenuation images of real size
        s = 1000.0 if "pcsd" in name else 1.0
        x = getattr(tigre.algorithms, name)(proj * np.float32(s), geo, ang, 3, tviter=5, **kw)
        assert np.isfinite(x).all(), name
        assert np.linalg.norm(x - s * img) < 0.8 * np.linalg.norm(s * img), name


def test_mlem_matches_oracle():
    """MLEM (statistical_algorithms.py:11-55): interpolated Ax, matched Atb, sensitivity image,
    multiplicative update, against the FP64 oracle restatement."""
    import tigre_b200 as tigre
    geo, ang, img = _case(views=24)
    proj = O.ax(img, geo, ang, "Siddon")
    got = tigre.algorithms.mlem(proj, geo, ang, 4)
    ref = O.mlem(proj, geo, ang, 4)
    mx, l2 = G.rel_err(got, ref)
    assert mx <= 1e-4 and l2 <= 1e-5, (mx, l2)
    x, res = tigre.algorithms.mlem(proj, geo, ang, 6, computel2=True)
    assert res.shape == (1, 6) and np.all(np.diff(res[0]) < 0)


@pytest.mark.parametrize("name", ["sart_tv", "ossart_tv"])
def test_sart_tv_first_iteration_matches_oracle_denoiser(name):
    """SART_TV / OSSART_TV (art_family_algorithms.py:65-152): one sweep, then im3ddenoise with
    the reference's tvlambda / tviter, against the oracle denoiser applied to the same sweep."""
    import tigre_b200 as tigre
    geo, ang, proj = _noisy_case()
    os_ = name == "ossart_tv"
    sweep = (tigre.algorithms.ossart(proj, geo, ang, 1, blocksize=5) if os_ else
             tigre.algorithms.sart(proj, geo, ang, 1))
    kw = {"blocksize": 5} if os_ else {}
    got = getattr(tigre.algorithms, name)(proj, geo, ang, 1, tviter=20, tvlambda=30, **kw)
    ref = O.im3ddenoise(sweep, 20, 30)
    mx, l2 = G.rel_err(got, ref)
    assert mx <= 1e-5 and l2 <= 1e-6, (name, mx, l2)


@pytest.mark.parametrize("name", ["hybrid_lsqr", "ab_gmres", "ba_gmres", "irn_tv_cgls"])
def test_krylov_extensions_match_oracle(name):
    """hybrid LSQR, AB-/BA-GMRES (matched backprojector), IRN-TV-CGLS against their FP64
    restatements over the oracle pair."""
    import tigre_b200 as tigre
    geo, ang, img = _case(views=24)
    proj = O.ax(img, geo, ang, "Siddon")
    if name == "hybrid_lsqr":
        ref, rl2 = O.hybrid_lsqr(proj, geo, ang, 6)
    elif name == "irn_tv_cgls":
        ref, rl2 = O.irn_tv_cgls(proj, geo, ang, 3, niter_outer=2)
    else:
        ref, rl2 = O.gmres(proj, geo, ang, 6, "proj" if name == "ab_gmres" else "vol")
    kw = {"niter_outer": 2} if name == "irn_tv_cgls" else {}
    n = 3 if name == "irn_tv_cgls" else 6
    got, l2 = getattr(tigre.algorithms, name)(proj, geo, ang, n, computel2=True, **kw)
    mx, e2 = G.rel_err(got, ref)
    assert mx <= 1e-3 and e2 <= 1e-4, (name, mx, e2)
    assert l2.shape[1] == len(rl2) and np.allclose(l2[0], rl2, rtol=1e-4), (l2, rl2)
    assert rl2[-1] < 0.5 * np.linalg.norm(proj)


def test_hybrid_flsqr_tv_matches_oracle():
    """hybrid fLSQR-TV against its FP64 restatement with scipy's LSQR for the inner solves."""
    import tigre_b200 as tigre
    geo, ang, img = _case(n=24, views=20)
    proj = O.ax(img, geo, ang, "Siddon")
    ref, rl2 = O.hybrid_flsqr_tv(proj, geo, ang, 4)
    got, l2 = tigre.algorithms.hybrid_flsqr_tv(proj, geo, ang, 4, computel2=True)
    mx, e2 = G.rel_err(got, ref)
    assert mx <= 1e-2 and e2 <= 1e-3, (mx, e2)
    assert np.allclose(l2[0], rl2, rtol=1e-3), (l2, rl2)
    assert rl2[-1] < 0.5 * np.linalg.norm(proj)


def test_gmres_fdk_backprojector_runs():
    import tigre_b200 as tigre
    geo, ang, img = _case(views=24)
    proj = O.ax(img, geo, ang, "Siddon")
    for name in ("ab_gmres", "ba_gmres"):
        x = getattr(tigre.algorithms, name)(proj, geo, ang, 4, backprojector="FDK")
        assert np.isfinite(x).all()
        assert np.linalg.norm(O.ax(x, geo, ang, "Siddon") - proj) < 0.5 * np.linalg.norm(proj), name


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
    """loss = |Ax - b|^2 + 1e-3 TV(x), central differences at h = 1e-3 along directions d.

    * TV term (hand-written backward): exact, checked along random directions;
    * data term: the backward of Ax is the matched backprojector, the reference's
      approximate adjoint of Siddon -- per voxel it differs for rough data, so the
      check is along smooth directions (Gaussian blobs), within its adjoint gap (<6% here)."""
    import torch
    from tigre_b200 import autograd as AG
    geo, ang, img = _case(n=24, views=18)
    rng = np.random.default_rng(0)
    A = AG.A(geo, ang)
    b = torch.from_numpy(O.ax(img, geo, ang, "Siddon")).cuda().double()
    x0 = torch.from_numpy((img + rng.normal(0, 5e-2, img.shape)).astype(np.float32)).cuda()
    h = 1e-3

    def data(x):
        r = A(x).double() - b
        return (r * r).sum()

    def tvl(x):
        return AG.tv(x).double()

    def loss(x):
        return data(x) + 1e-3 * tvl(x)

    def grad(f):
        x = x0.clone().requires_grad_(True)
        f(x).backward()
        return x.grad.double()

    def fd(f, d):
        return (f(x0 + h * d) - f(x0 - h * d)).item() / (2 * h)

    zz, yy, xx = np.meshgrid(*[np.arange(24)] * 3, indexing="ij")
    blobs = []
    for c in [(12, 12, 12), (8, 15, 10), (16, 6, 9)]:
        blob = np.exp(-((zz - c[0]) ** 2 + (yy - c[1]) ** 2 + (xx - c[2]) ** 2) / (2 * 3.0 ** 2))
        blobs.append(torch.from_numpy(blob.astype(np.float32)).cuda())
    g_data, g_all = grad(data), grad(loss)
    for d in blobs:
        e_data = abs(fd(data, d) - (g_data * d).sum().item()) / abs(fd(data, d))
        e_all = abs(fd(loss, d) - (g_all * d).sum().item()) / abs(fd(loss, d))
        assert e_data < 0.06 and e_all < 0.06, (e_data, e_all)
    # TV along random directions.  |grad f| has curvature ~1/|grad f|, so the step is small
    # and the quotient uses the FP64 TV sum (the loss value itself is FP32); the volume is
    # shifted by +4 so that the zero-halo terms |f| of the top slice stay off their kink at 0
    from tigre_b200 import projectors as P
    x1 = x0 + 4.0
    g1 = P.tv_gradient(x1).double()
    for seed in range(3):
        d = torch.from_numpy(np.random.default_rng(seed).normal(0, 1, img.shape).astype(np.float32)).cuda()
        ref = (P.tv_value(x1 + 1e-4 * d).item() - P.tv_value(x1 - 1e-4 * d).item()) / 2e-4
        assert abs(ref - (g1 * d).sum().item()) <= 2e-3 * abs(ref), (seed, ref)
    x = x1.clone().requires_grad_(True)
    tvl(x).backward()
    torch.testing.assert_close(x.grad.double(), g1)


def test_autograd_batch_dimension():
    import torch
    from tigre_b200 import autograd as AG, projectors as P
    geo, ang, img = _case()
    A = AG.A(geo, ang)
    xb = torch.stack([torch.from_numpy(img), torch.from_numpy(img[::-1].copy())]).cuda()
    yb = A(xb)
    assert yb.shape == (2, 24, 48, 64)
    torch.testing.assert_close(yb[1], P.ax(xb[1].contiguous(), A.plan, "Siddon"))


@pytest.mark.parametrize("filt", [None, "hann"])
def test_fbp_parallel_matches_oracle(filt):
    """Parallel-beam FBP (single_pass_algorithms.py:206-228) against the oracle's host-side
    filter and parallel backprojection; it also reconstructs the phantom."""
    import tigre_b200 as tigre
    from tigre_b200.utilities.geometry import geometry
    geo = geometry(mode="parallel", nVoxel=np.array([24, 40, 40]))
    ang = np.linspace(0, np.pi, 120, endpoint=False).astype(np.float32)
    img = G.phantom((24, 40, 40), seed=13)
    proj = O.ax(img, geo, ang, "Siddon")
    got = tigre.algorithms.fbp(proj, geo, ang, filter=filt)
    ref = O.fbp(proj, geo, ang, filt)
    mx, l2 = G.rel_err(got, ref)
    assert mx <= 2e-5 and l2 <= 1e-5, (mx, l2)
    if filt is None:
        assert np.linalg.norm(got - img) / np.linalg.norm(img) < 0.35
    with pytest.raises(ValueError):
        tigre.algorithms.fbp(proj, G.c1_geometry(), ang)


@pytest.mark.parametrize("name", ["lsqr", "lsmr"])
def test_lsqr_lsmr_match_oracle(name):
    """LSQR / LSMR (krylov_subspace_algorithms.py:101-187, :299-439) against the same
    recurrences in FP64 over the oracle pair; residuals decrease."""
    import tigre_b200 as tigre
    geo, ang, img = _case()
    proj = O.ax(img, geo, ang, "Siddon")
    x, l2 = getattr(tigre.algorithms, name)(proj, geo, ang, 6, computel2=True)
    xr, resr = getattr(O, name)(proj, geo, ang, 6)
    mx, l2e = G.rel_err(x, xr)
    assert l2e <= 1e-4, (name, mx, l2e)
    np.testing.assert_allclose(l2.ravel()[:len(resr)], resr, rtol=1e-4)
    assert np.all(np.diff(l2.ravel()) < 0)


def test_fista_matches_oracle_and_ista_runs():
    """FISTA (ista_algorithms.py:13-176) against the same steps in FP64 over the oracle pair
    and the oracle TV denoiser; ISTA returns a finite, nonnegative-clipped volume."""
    import tigre_b200 as tigre
    geo, ang, img = _case(n=24, views=18)
    proj = O.ax(img, geo, ang, "interpolated")
    hyper = 4.0e5
    got = tigre.algorithms.fista(proj, geo, ang, 3, hyper=hyper, tviter=10)
    ref = O.fista(proj, geo, ang, 3, hyper, tviter=10)
    mx, l2 = G.rel_err(got, ref)
    assert mx <= 1e-4 and l2 <= 1e-5, (mx, l2)
    x, l2s = tigre.algorithms.ista(proj, geo, ang, 2, hyper=hyper, computel2=True)
    assert np.isfinite(x).all() and l2s.shape == (1, 2)


def test_quameasopts_reporting():
    """Quameasopts (iterative_recon_alg.py:205-209, :362-364): per iteration, the quality
    measures between the new and the previous iterate; with computel2 the residual row comes
    first (geterrors, :406-410)."""
    import tigre_b200 as tigre
    from tigre_b200.utilities.Measure_Quality import Measure_Quality
    geo, ang, img = _case(views=20)
    proj = O.ax(img, geo, ang, "Siddon")
    x, err = tigre.algorithms.ossart(proj, geo, ang, 3, blocksize=5, Quameasopts=["RMSE", "CC"], computel2=True)
    assert err.shape == (3, 3) and np.all(np.diff(err[0]) < 0)
    x1 = tigre.algorithms.ossart(proj, geo, ang, 1, blocksize=5)
    x2 = tigre.algorithms.ossart(proj, geo, ang, 2, blocksize=5)
    np.testing.assert_allclose(err[1:, 1], Measure_Quality(x2, x1, ["RMSE", "CC"]), rtol=1e-4)
    xc, q = tigre.algorithms.cgls(proj, geo, ang, 4, Quameasopts="RMSE")
    assert q.shape == (1, 4) and np.all(q > 0)
