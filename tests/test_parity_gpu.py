"""Parity of the sm_100a projector pair with the FP64 oracle, through the C ABI.

Bar (FP32 storage, FP64 geometry, exact interpolation): max|gpu-oracle| / max|oracle|
and ||gpu-oracle|| / ||oracle|| both <= TOL = 1e-5.
"""
import numpy as np
import pytest

from tests import geometries as G
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _torch():
    import torch
    return torch


CASES = {
    "c1": (G.c1_geometry, lambda: G.angles(100), 0),
    "odd": (G.odd_geometry, lambda: G.angles(37, full=np.pi * 1.3), 1),
    "tilted": (G.tilted_geometry, lambda: G.angles(23, tilt=True), 2),
    "steep": (G.steep_geometry, lambda: G.angles(29), 3),
}


@pytest.fixture(scope="module", params=list(CASES))
def case(request):
    mk_geo, mk_ang, seed = CASES[request.param]
    geo = mk_geo()
    ang = mk_ang()
    img = G.phantom(tuple(int(v) for v in geo.nVoxel), seed=seed)
    return request.param, geo, ang, img


@pytest.mark.parametrize("ptype", ["Siddon", "interpolated"])
def test_ax_host_api_matches_oracle(case, ptype):
    import tigre_b200 as tigre
    name, geo, ang, img = case
    got = tigre.Ax(img, geo, ang, ptype)
    ref = O.ax(img, geo, ang, ptype)
    mx, l2 = G.rel_err(got, ref)
    assert mx <= TOL and l2 <= TOL, (name, ptype, mx, l2)


@pytest.mark.parametrize("btype", ["FDK", "matched"])
def test_atb_host_api_matches_oracle(case, btype):
    import tigre_b200 as tigre
    name, geo, ang, img = case
    proj = O.ax(img, geo, ang, "Siddon")
    got = tigre.Atb(proj, geo, ang, btype)
    ref = O.atb(proj, geo, ang, btype)
    mx, l2 = G.rel_err(got, ref)
    assert mx <= TOL and l2 <= TOL, (name, btype, mx, l2)


@pytest.mark.parametrize("ptype", ["Siddon", "interpolated"])
def test_device_api_equals_host_api(case, ptype):
    torch = _torch()
    import tigre_b200 as tigre
    name, geo, ang, img = case
    host = tigre.Ax(img, geo, ang, ptype)
    dev = tigre.Ax(torch.from_numpy(img).cuda(), geo, ang, ptype).cpu().numpy()
    np.testing.assert_array_equal(dev, host)


def test_device_atb_equals_host(case):
    torch = _torch()
    import tigre_b200 as tigre
    name, geo, ang, img = case
    proj = O.ax(img, geo, ang, "Siddon")
    for bt in ("FDK", "matched"):
        host = tigre.Atb(proj, geo, ang, bt)
        dev = tigre.Atb(torch.from_numpy(proj).cuda(), geo, ang, bt).cpu().numpy()
        np.testing.assert_array_equal(dev, host)


def test_siddon_segment_count_matches_oracle():
    torch = _torch()
    from tigre_b200 import _native as N, projectors
    geo, ang = G.c1_geometry(), G.angles(20)
    img = G.phantom((64, 64, 64))
    _, cnt = O.ax(img, geo, ang, "Siddon", return_counts=True)
    plan = N.get_plan(N.checked_geometry(geo, ang), 0)
    total = projectors.siddon_segments(plan)
    # the oracle skips zero-length segments at exact edge crossings
    assert abs(total - int(cnt.sum())) <= 1e-4 * int(cnt.sum()), (total, int(cnt.sum()))


@pytest.mark.parametrize("tilt", [False, True])
def test_interp_sample_count_matches_oracle(tilt):
    """tigre_interp_count_samples against the oracle's per-ray sample counts (samples strictly
    inside the open box), axial and with theta/psi rotations (the spherical cap)."""
    _torch()
    from tigre_b200 import _native as N, projectors
    geo, ang = G.c1_geometry(), G.angles(20, tilt=tilt)
    img = G.phantom((64, 64, 64))
    _, cnt = O.ax(img, geo, ang, "interpolated", return_counts=True)
    plan = N.get_plan(N.checked_geometry(geo, ang), 0)
    total = projectors.interp_samples(plan)
    ref = int(cnt.sum())
    # boundary samples whose coordinate rounds onto -1 or n may fall either way
    assert ref > 0 and abs(total - ref) <= 1e-4 * ref, (total, ref)


def test_angle_subrange_matches_full():
    torch = _torch()
    from tigre_b200 import _native as N, projectors
    geo, ang = G.c1_geometry(), G.angles(40)
    img = torch.from_numpy(G.phantom((64, 64, 64))).cuda()
    plan = N.get_plan(N.checked_geometry(geo, ang), 0)
    full = projectors.ax(img, plan, "Siddon")
    part = projectors.ax(img, plan, "Siddon", angle_range=(13, 29))
    torch.testing.assert_close(part, full[13:29], rtol=0, atol=0)
    bp_full = projectors.atb(full[13:29].contiguous(), plan, "matched", angle_range=(13, 29))
    ref = O.atb(full.cpu().numpy(), geo, ang, "matched", angle_range=(13, 29))
    mx, l2 = G.rel_err(bp_full.cpu().numpy(), ref)
    assert mx <= TOL and l2 <= TOL


def test_tv_gradient_and_pocs_match_oracle():
    torch = _torch()
    from tigre_b200 import projectors
    rng = np.random.default_rng(5)
    img = (G.phantom((24, 31, 29), seed=4) + rng.normal(0, 1e-3, (24, 31, 29))).astype(np.float32)
    g = projectors.tv_gradient(torch.from_numpy(img).cuda()).cpu().numpy()
    gref = O.tv_gradient(img)
    mx, l2 = G.rel_err(g, gref)
    assert mx <= 1e-4 and l2 <= TOL, (mx, l2)
    import tigre_b200 as tigre
    out = tigre.minTV(img, alpha=0.002, maxiter=20)
    ref = O.pocs_tv(img, 0.002, 20)
    mx, l2 = G.rel_err(out, ref)
    assert mx <= TOL and l2 <= TOL, (mx, l2)


@pytest.mark.parametrize("shape", [(24, 31, 29), (1, 17, 13), (2, 9, 40)])
def test_awtv_matches_oracle(shape):
    """AwminTV (aw_pocs_tv, GD_AwTV.cu:276): host entry point and device path against the
    oracle, at the default delta and at one of the order of the differences."""
    torch = _torch()
    import tigre_b200 as tigre
    rng = np.random.default_rng(21)
    img = (G.phantom(shape, seed=21) + rng.normal(0, 1e-3, shape)).astype(np.float32)
    for delta in (-0.005, 0.02):
        ref = O.aw_pocs_tv(img, 0.002, 15, delta)
        out = tigre.AwminTV(img, alpha=0.002, maxiter=15, delta=delta)
        mx, l2 = G.rel_err(out, ref)
        assert mx <= TOL and l2 <= TOL, ("host", delta, mx, l2)
        dev = tigre.AwminTV(torch.from_numpy(img).cuda(), alpha=0.002, maxiter=15, delta=delta).cpu().numpy()
        mx, l2 = G.rel_err(dev, ref)
        assert mx <= TOL and l2 <= TOL, ("device", delta, mx, l2)


@pytest.mark.parametrize("shape", [(24, 31, 29), (1, 17, 13), (3, 8, 33)])
def test_piccs_matches_oracle(shape):
    """minPICCS (piccs_tv, PICCS.cu:274): host entry point and device path against the oracle."""
    torch = _torch()
    import tigre_b200 as tigre
    from tests import golden_cases as GC
    rng = np.random.default_rng(22)
    img = (G.phantom(shape, seed=22) + rng.normal(0, 1e-3, shape)).astype(np.float32)
    prior = GC.piccs_prior(img)
    for ratio in (0.95, 0.5):
        ref = O.piccs_tv(img, prior, 0.002, ratio, 15)
        out = tigre.minPICCS(img, prior, alpha=0.002, maxiter=15, ratio=ratio)
        mx, l2 = G.rel_err(out, ref)
        assert mx <= TOL and l2 <= TOL, ("host", ratio, mx, l2)
        dev = tigre.minPICCS(torch.from_numpy(img).cuda(), torch.from_numpy(prior).cuda(), alpha=0.002, maxiter=15,
                             ratio=ratio).cpu().numpy()
        mx, l2 = G.rel_err(dev, ref)
        assert mx <= TOL and l2 <= TOL, ("device", ratio, mx, l2)


def test_tv_value_consistent_with_gradient():
    """Central differences of tv_value reproduce tv_gradient (noisy volume, |grad| >> eps)."""
    torch = _torch()
    from tigre_b200 import projectors
    rng = np.random.default_rng(7)
    # offset keeps the zero-halo terms |f| away from their kink at 0
    x = torch.from_numpy((rng.normal(0, 1, (6, 7, 8)) + 4.0).astype(np.float32)).cuda()
    g = projectors.tv_gradient(x).cpu().numpy().astype(np.float64)
    h = 1e-3
    idx = [(0, 0, 0), (5, 6, 7), (2, 3, 4), (5, 0, 3), (0, 6, 7)]
    for (z, y, xx) in idx:
        xp = x.clone(); xp[z, y, xx] += h
        xm = x.clone(); xm[z, y, xx] -= h
        fd = (projectors.tv_value(xp).item() - projectors.tv_value(xm).item()) / (2 * h)
        assert abs(fd - g[z, y, xx]) <= 5e-3 * max(1.0, abs(g[z, y, xx])), ((z, y, xx), fd, g[z, y, xx])


def test_bf16_storage_error_is_small():
    """Reduced-precision storage: stated error against the FP64 oracle (bound 1e-2)."""
    torch = _torch()
    from tigre_b200 import _native as N, projectors
    geo, ang = G.c1_geometry(), G.angles(50)
    img = G.phantom((64, 64, 64))
    plan = N.get_plan(N.checked_geometry(geo, ang), 0)
    ref = O.ax(img, geo, ang, "Siddon")
    for dt in (torch.bfloat16, torch.float16):
        p = projectors.ax(torch.from_numpy(img).cuda().to(dt), plan, "Siddon", out_dtype=torch.float32)
        mx, l2 = G.rel_err(p.cpu().numpy(), ref)
        assert l2 <= 1e-2, (dt, mx, l2)


def test_adjoint_dot_test_matched():
    """<Ax, y> vs <x, A^T y> for Siddon + matched; the matched weight is the reference's
    approximate adjoint, so the gap is reported and bounded loosely (2%)."""
    torch = _torch()
    from tigre_b200 import _native as N, projectors
    geo, ang = G.c1_geometry(), G.angles(60)
    rng = np.random.default_rng(11)
    x = torch.from_numpy(rng.random((64, 64, 64), dtype=np.float32)).cuda()
    y = torch.from_numpy(rng.random((60, 128, 128), dtype=np.float32)).cuda()
    plan = N.get_plan(N.checked_geometry(geo, ang), 0)
    ax = projectors.ax(x, plan, "Siddon")
    aty = projectors.atb(y, plan, "matched")
    lhs = float((ax.double() * y.double()).sum())
    rhs = float((x.double() * aty.double()).sum())
    assert abs(lhs - rhs) / abs(lhs) < 0.02, (lhs, rhs)


def test_empty_and_missing_rays():
    """Views whose rays miss the volume entirely give exact zeros (reference writes 0)."""
    torch = _torch()
    import tigre_b200 as tigre
    geo = G.c1_geometry()
    geo.offOrigin = np.array((500.0, 0.0, 0.0))    # volume moved 500 mm along z, out of the cone
    img = G.phantom((64, 64, 64))
    p = tigre.Ax(img, geo, G.angles(4), "Siddon")
    assert np.all(p == 0)
    q = tigre.Ax(img, geo, G.angles(4), "interpolated")
    assert np.all(q == 0)


def test_staged_backprojector_fallback_and_status():
    """Blocks whose footprint does not fit the shared-memory box take the bounds-checked
    global path; both paths agree with the oracle and leave the status word clean."""
    import torch
    from tigre_b200 import _native as N, projectors as P
    geo, ang = G.c1_geometry(), G.angles(30)
    img = G.phantom((64, 64, 64))
    proj = O.ax(img, geo, ang, "Siddon")
    with N.option(N.OPT_BP_BOX, (8 << 16) | 4):
        plan = N.get_plan(N.checked_geometry(geo, ang), 0)
        for bt in ("FDK", "matched"):
            got = P.atb(torch.from_numpy(proj).cuda(), plan, bt).cpu().numpy()
            mx, l2 = G.rel_err(got, O.atb(proj, geo, ang, bt))
            assert mx <= TOL and l2 <= TOL, (bt, mx, l2)
        assert plan.status() == 0


def test_plain_backprojector_matches_oracle(case):
    """The global-load backprojector (used for FP16 projections, and selected here for FP32
    with TIGRE_OPT_BP_KERNEL) meets the same bar as the TMA-staged one."""
    import torch
    from tigre_b200 import _native as N, projectors as P
    name, geo, ang, img = case
    proj = O.ax(img, geo, ang, "Siddon")
    with N.option(N.OPT_BP_KERNEL, 1):
        plan = N.get_plan(N.checked_geometry(geo, ang), 0)
        for bt in ("FDK", "matched"):
            got = P.atb(torch.from_numpy(proj).cuda(), plan, bt).cpu().numpy()
            mx, l2 = G.rel_err(got, O.atb(proj, geo, ang, bt))
            assert mx <= TOL and l2 <= TOL, (name, bt, mx, l2)
        assert plan.status() == 0


def test_status_word_clean_after_projectors(case):
    import torch
    from tigre_b200 import _native as N, projectors as P
    name, geo, ang, img = case
    plan = N.get_plan(N.checked_geometry(geo, ang), 0)
    p = P.ax(torch.from_numpy(img).cuda(), plan, "Siddon")
    P.atb(p, plan, "FDK")
    P.atb(p, plan, "matched")
    assert plan.status() == 0


def test_atb_accumulate_over_view_chunks(case):
    """tigre_atb_ex with accumulate: the sum of chunk backprojections equals one call."""
    import ctypes as C
    import torch
    from tigre_b200 import _native as N, projectors as P
    name, geo, ang, img = case
    plan = N.get_plan(N.checked_geometry(geo, ang), 0)
    proj = P.ax(torch.from_numpy(img).cuda(), plan, "Siddon")
    L = N.lib()
    for bt in (N.BACKPROJ_FDK, N.BACKPROJ_MATCHED):
        full = P.atb(proj, plan, "matched" if bt else "FDK")
        acc = torch.full_like(full, float("nan"))
        n, k = proj.shape[0], proj.shape[0] // 3
        stream = torch.cuda.current_stream().cuda_stream
        for j, (a, b) in enumerate(((0, k), (k, 2 * k), (2 * k, n))):
            N.check(L.tigre_atb_ex(plan.handle, proj[a:b].data_ptr(), N.F32, acc.data_ptr(), N.F32, bt, a, b,
                                   int(j > 0), C.c_void_p(stream)), "tigre_atb_ex")
        mx, l2 = G.rel_err(acc.cpu().numpy(), full.cpu().numpy())
        assert mx <= 1e-5 and l2 <= 1e-6, (name, bt, mx, l2)
    assert plan.status() == 0


def test_host_pipeline_with_small_chunks():
    """The host entry points stream views through two device buffers; with 4-view chunks
    (and a last partial chunk) the results equal the single-chunk call and the oracle."""
    import tigre_b200 as tigre
    from tigre_b200 import _native as N
    geo, ang = G.odd_geometry(), G.angles(23, full=np.pi * 1.3)
    img = G.phantom(tuple(int(v) for v in geo.nVoxel), seed=5)
    with N.option(N.OPT_HOST_CHUNK_VIEWS, 4):
        for _ in range(2):
            p = tigre.Ax(img, geo, ang, "Siddon")
            r = O.ax(img, geo, ang, "Siddon")
            mx, l2 = G.rel_err(p, r)
            assert mx <= TOL and l2 <= TOL, ("ax", mx, l2)
            for bt in ("FDK", "matched"):
                v = tigre.Atb(r, geo, ang, bt)
                mx, l2 = G.rel_err(v, O.atb(r, geo, ang, bt))
                assert mx <= TOL and l2 <= TOL, (bt, mx, l2)


@pytest.mark.parametrize("kernel", [1, 2])
def test_other_siddon_kernels_match_oracle(kernel):
    """TIGRE_OPT_SIDDON_KERNEL 1 keeps the stepped column kernel (one-crossing variant) and 2
    the generic per-ray kernel on the axial geometries; both meet the bar of the default
    cell-interval kernel."""
    import torch
    from tigre_b200 import _native as N, projectors as P
    with N.option(N.OPT_SIDDON_KERNEL, kernel):
        for mk, ang in ((G.c1_geometry, G.angles(40)), (G.odd_geometry, G.angles(23, full=np.pi * 1.3))):
            geo = mk()
            img = G.phantom(tuple(int(v) for v in geo.nVoxel), seed=4)
            plan = N.get_plan(N.checked_geometry(geo, ang), 0)
            got = P.ax(torch.from_numpy(img).cuda(), plan, "Siddon").cpu().numpy()
            mx, l2 = G.rel_err(got, O.ax(img, geo, ang, "Siddon"))
            assert mx <= TOL and l2 <= TOL, (kernel, mx, l2)
            assert plan.status() == 0


@pytest.mark.parametrize("dt", ["bfloat16", "float16"])
def test_reduced_storage_equals_fp32_on_rounded_inputs(dt):
    """BF16 / FP16 storage changes only what is stored: each projector kind run on 16-bit
    inputs (FP32 output) equals the FP32 path run on the same inputs rounded to 16 bits."""
    torch = _torch()
    from tigre_b200 import _native as N, projectors as P
    tdt = getattr(torch, dt)
    geo, ang = G.odd_geometry(), G.angles(17, full=np.pi * 1.3)
    img = G.phantom(tuple(int(v) for v in geo.nVoxel), seed=9)
    plan = N.get_plan(N.checked_geometry(geo, ang), 0)
    v16 = torch.from_numpy(img).cuda().to(tdt)
    v32 = v16.float()
    for ptype in ("Siddon", "interpolated"):
        got = P.ax(v16, plan, ptype, out_dtype=torch.float32).cpu().numpy()
        ref = P.ax(v32, plan, ptype).cpu().numpy()
        mx, l2 = G.rel_err(got, ref)
        assert mx <= 1e-5 and l2 <= 1e-6, (dt, ptype, mx, l2)
    p16 = torch.from_numpy(O.ax(img, geo, ang, "Siddon")).cuda().to(tdt)
    p32 = p16.float()
    for bt in ("FDK", "matched"):
        got = P.atb(p16, plan, bt, out_dtype=torch.float32).cpu().numpy()
        ref = P.atb(p32, plan, bt).cpu().numpy()
        mx, l2 = G.rel_err(got, ref)
        assert mx <= 1e-5 and l2 <= 1e-6, (dt, bt, mx, l2)
    assert plan.status() == 0


def test_interpolated_point_sampling_matches_oracle():
    """accuracy > 1 switches the interpolated projector to point sampling (the reference's
    texture switches to cudaFilterModePoint, ray_interpolated_projection.cu:589-592).

    Point sampling is discontinuous where a sample crosses a voxel half-boundary: the sample
    positions are FP32 here (as in the reference), FP64 in the oracle, so a sample within
    ~1e-4 voxel of a boundary may pick the neighbouring voxel.  Such a ray differs by one
    sample's value; every other ray must agree to the parity bar."""
    torch = _torch()
    from tigre_b200 import _native as N, projectors as P
    geo, ang = G.c1_geometry(), G.angles(24)
    geo.accuracy = 2.0
    img = G.phantom((64, 64, 64), seed=6)
    plan = N.get_plan(N.checked_geometry(geo, ang), 0)
    got = P.ax(torch.from_numpy(img).cuda(), plan, "interpolated").cpu().numpy().astype(np.float64)
    ref = O.ax(img, geo, ang, "interpolated").astype(np.float64)
    err = np.abs(got - ref) / np.abs(ref).max()
    bad = err > TOL
    # one flipped sample changes a ray by at most (max voxel) x (sample length in mm)
    one_sample = float(img.max()) * 2.0 * 1.0 / np.abs(ref).max()
    assert bad.mean() <= 2e-3, (bad.mean(), err.max())
    assert err.max() <= 2.0 * one_sample, (err.max(), one_sample)


def _parallel_case():
    from tigre_b200.utilities.geometry import geometry
    geo = geometry(mode="parallel", nVoxel=np.array([36, 44, 40]))
    geo.offOrigin = np.array((1.5, -2.0, 0.75))
    geo.offDetector = np.array((0.8, -1.2))
    geo.COR = -0.4
    ang = G.angles(19, full=np.pi)
    img = G.phantom((36, 44, 40), seed=12)
    return geo, ang, img


@pytest.mark.parametrize("ptype", ["Siddon", "interpolated"])
def test_parallel_projection_matches_oracle(ptype):
    """Parallel beam (siddon_ray_projection_parallel / interpolation_projection_parallel):
    host and device APIs against the FP64 oracle, with origin and detector offsets and COR."""
    torch = _torch()
    import tigre_b200 as tigre
    from tigre_b200 import _native as N, projectors as P
    geo, ang, img = _parallel_case()
    ref = O.ax(img, geo, ang, ptype)
    got = tigre.Ax(img, geo, ang, ptype)
    mx, l2 = G.rel_err(got, ref)
    assert mx <= TOL and l2 <= TOL, ("host", ptype, mx, l2)
    plan = N.get_plan(N.checked_geometry(geo, ang), 0)
    assert plan.parallel
    dev = P.ax(torch.from_numpy(img).cuda(), plan, ptype).cpu().numpy()
    mx, l2 = G.rel_err(dev, ref)
    assert mx <= TOL and l2 <= TOL, ("device", ptype, mx, l2)
    assert plan.status() == 0


def test_parallel_backprojection_matches_oracle():
    """voxel_backprojection_parallel: orthographic, unit weight; the backprojection type is
    ignored in parallel beam, as in the reference."""
    torch = _torch()
    import tigre_b200 as tigre
    from tigre_b200 import _native as N, projectors as P
    geo, ang, img = _parallel_case()
    proj = O.ax(img, geo, ang, "Siddon")
    ref = O.atb(proj, geo, ang, "FDK")
    for bt in ("FDK", "matched"):
        got = tigre.Atb(proj, geo, ang, bt)
        mx, l2 = G.rel_err(got, ref)
        assert mx <= TOL and l2 <= TOL, ("host", bt, mx, l2)
    plan = N.get_plan(N.checked_geometry(geo, ang), 0)
    dev = P.atb(torch.from_numpy(proj).cuda(), plan, "matched").cpu().numpy()
    mx, l2 = G.rel_err(dev, ref)
    assert mx <= TOL and l2 <= TOL, ("device", mx, l2)
    assert plan.status() == 0


def test_tv_denoise_matches_oracle():
    """im3ddenoise / tvdenoising (tv_proximal.cu:185-630): host entry point and device path
    against the FP64 oracle restatement, including the min/max scaling of im_3d_denoise.py."""
    torch = _torch()
    from tigre_b200.utilities.im_3d_denoise import im3ddenoise, tv_denoise_device
    rng = np.random.default_rng(17)
    img = (G.phantom((21, 34, 27), seed=17) + rng.normal(0, 0.003, (21, 34, 27))).astype(np.float32)
    ref = O.im3ddenoise(img, 25, 12.0)
    got = im3ddenoise(img, 25, 12.0)
    mx, l2 = G.rel_err(got, ref)
    assert mx <= TOL and l2 <= TOL, ("host", mx, l2)
    dev = im3ddenoise(torch.from_numpy(img).cuda(), 25, 12.0).cpu().numpy()
    mx, l2 = G.rel_err(dev, ref)
    assert mx <= TOL and l2 <= TOL, ("device", mx, l2)
    # unscaled device operator on a single slice and on two slices (edge of the z halo rule)
    for nz in (1, 2):
        x = np.ascontiguousarray(img[:nz])
        out = tv_denoise_device(torch.from_numpy(x).cuda(), 10, 5.0).cpu().numpy()
        mx, l2 = G.rel_err(out, O.tvdenoise(x, 10, 5.0))
        assert mx <= TOL and l2 <= TOL, (nz, mx, l2)


@pytest.mark.parametrize("nv", [300, 520])
def test_siddon_tall_detectors(nv):
    """Tall detectors select 4 (nV >= 256) or 8 (nV >= 512) rows per thread in the
    cell-interval kernel; partial row tiles included."""
    torch = _torch()
    from tigre_b200 import _native as N, projectors as P
    from tigre_b200.utilities.geometry import cone_geometry
    geo = cone_geometry((40, 36, 36), (40.0, 36.0, 36.0), (nv, 28), (0.1, 1.6))
    ang = G.angles(5)
    img = G.phantom((40, 36, 36), seed=14)
    plan = N.get_plan(N.checked_geometry(geo, ang), 0)
    got = P.ax(torch.from_numpy(img).cuda(), plan, "Siddon").cpu().numpy()
    mx, l2 = G.rel_err(got, O.ax(img, geo, ang, "Siddon"))
    assert mx <= TOL and l2 <= TOL, (nv, mx, l2)
    assert plan.status() == 0


def test_full_size_parity_on_subsets():
    """The metric workload itself (512^3 @ 0.5 mm, 1024x768 @ 0.4 mm, 720 views over 2 pi, DSO
    1000, DSD 1536): rows of three views of the Siddon and interpolated projections, and two
    slices of the matched and FDK backprojections of all 720 views, against the oracle."""
    torch = _torch()
    from tigre_b200 import _native as N, projectors as P
    from tigre_b200.utilities.geometry import cone_geometry
    from tigre_b200.utilities.phantom import random_ellipsoids
    geo = cone_geometry((512, 512, 512), (256.0, 256.0, 256.0), (768, 1024), (0.4, 0.4))
    ang = np.zeros((720, 3), dtype=np.float32)
    ang[:, 0] = np.linspace(0, 2 * np.pi, 720, endpoint=False)
    img = random_ellipsoids((512, 512, 512), seed=0, device="cuda")
    plan = N.get_plan(N.checked_geometry(geo, ang), 0)
    img_h = img.cpu().numpy()
    proj = P.ax(img, plan, "Siddon")
    for ptype in ("Siddon", "interpolated"):
        p = proj if ptype == "Siddon" else P.ax(img, plan, "interpolated")
        for a, r0 in ((0, 380), (137, 10), (541, 700)):
            ref = O.ax(img_h, geo, ang, ptype, angle_range=(a, a + 1), row_range=(r0, r0 + 8))
            got = p[a:a + 1, r0:r0 + 8].cpu().numpy()
            mx, l2 = G.rel_err(got, ref)
            assert mx <= TOL and l2 <= TOL, (ptype, a, r0, mx, l2)
        del p
    proj_h = proj.cpu().numpy()
    for btype in ("matched", "FDK"):
        bp = P.atb(proj, plan, btype)
        for z0 in (3, 255):
            ref = O.atb(proj_h, geo, ang, btype, z_range=(z0, z0 + 2))
            mx, l2 = G.rel_err(bp[z0:z0 + 2].cpu().numpy(), ref)
            assert mx <= TOL and l2 <= TOL, (btype, z0, mx, l2)
        del bp


@pytest.mark.parametrize("name", ["small", "offsets", "rotated", "c1"])
def test_texture_interpolation_against_reference_and_oracle(name):
    """TIGRE_OPT_INTERP_TEXTURE: the interpolated projector sampling through the texture unit
    (8-bit filter weights, as the reference's own projector).  Against the reference's output
    (golden fixtures made by its CUDA build) it agrees to the texture quantisation; against the
    exact FP64 oracle it stays within the reference's own distance from it (5e-3 max, 5e-4 L2)."""
    import os
    import torch
    from tests import golden_cases as GC
    from tigre_b200 import _native as N, projectors as P
    geo, ang, img = GC.make(name)
    ref = np.load(os.path.join(os.path.dirname(__file__), "golden", "ref_%s.npz" % name))["interpolated"]
    with N.option(N.OPT_INTERP_TEXTURE, 1):
        plan = N.get_plan(N.checked_geometry(geo, ang), 0)
        got = P.ax(torch.from_numpy(img).cuda(), plan, "interpolated").cpu().numpy()
    exact = O.ax(img, geo, ang, "interpolated")
    mx_r, l2_r = G.rel_err(got, ref)
    mx_o, l2_o = G.rel_err(got, exact)
    print("%s: texture vs reference max %.2e L2 %.2e; vs FP64 oracle max %.2e L2 %.2e" % (name, mx_r, l2_r, mx_o, l2_o))
    assert mx_o <= 5e-3 and l2_o <= 5e-4, (mx_o, l2_o)
    assert l2_r <= l2_o, (l2_r, l2_o)    # closer to the reference than to exact interpolation
