"""The FP64 oracle against outputs of the reference's own CUDA build (tests/golden/,
made by tests/golden/make_golden.py on a B200).

Tolerances are the reference's own precision, not the 1e-5 bar of our kernels:
its Siddon traverses in FP32 alpha from the source with __fdividef/__frcp_rd
(Siddon_projection.cu:168-266); its interpolated projector and backprojectors
sample textures with 8-bit fractional weights (ray_interpolated_projection.cu:594,
voxel_backprojection.cu:707); pocs_tv has no interpolation and agrees tightly.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O
from tests import golden_cases as GC
from tests.geometries import rel_err

HERE = os.path.dirname(os.path.abspath(__file__))

# (max-abs / max-ref, L2-relative) per output
TOLS = {
    "siddon": (5e-4, 1e-4),
    "interpolated": (5e-3, 5e-4),
    "fdk": (2e-3, 2e-4),
    "matched": (2e-3, 2e-4),
    "pocs_tv": (1e-5, 1e-6),
    "tvdenoise": (1e-5, 1e-6),
    "awtv": (1e-5, 1e-6),
    # piccs_tv sums |g|^2 in FP32 (reduceNorm2/reduceSum, PICCS.cu:352-366): up to ~1e-5 of drift
    "piccs": (2e-5, 1e-6),
}


def _oracle_output(key, img, geo, ang, ref):
    if key == "siddon":
        return O.ax(img, geo, ang, "Siddon")
    if key == "interpolated":
        return O.ax(img, geo, ang, "interpolated")
    if key in ("fdk", "matched"):
        return O.atb(ref["siddon"], geo, ang, "FDK" if key == "fdk" else "matched")
    if key == "pocs_tv":
        return O.pocs_tv(img, GC.TV_ALPHA, GC.TV_ITERS)
    if key == "tvdenoise":
        return O.tvdenoise((img - img.min()) / (img - img.min()).max(), GC.DENOISE_ITERS, GC.DENOISE_LAMBDA)
    if key == "awtv":
        return O.aw_pocs_tv(img, GC.TV_ALPHA, GC.TV_ITERS, GC.AWTV_DELTA)
    if key == "piccs":
        return O.piccs_tv(img, GC.piccs_prior(img), GC.TV_ALPHA, GC.PICCS_RATIO, GC.TV_ITERS)
    raise KeyError(key)


# Rays on which the reference's own Siddon output is wrong: (case, view, detector column).  On
# the C1-size case every row of column 69 of view 2 (64.8 degrees) misses or gains part of its
# line integral (up to 5.9 % of the maximum; 95 of 196,608 rays); an independent fine-sampled
# line integral agrees with the oracle there (test below), so these rays are excluded from the
# comparison -- and the exclusion must stay exactly this set.
REFERENCE_SIDDON_DEFECTS = {"c1": [(2, 69)]}


def _defect_mask(name, shape):
    mask = np.zeros(shape, dtype=bool)
    for view, col in REFERENCE_SIDDON_DEFECTS.get(name, []):
        mask[view, :, col] = True
    return mask


@pytest.mark.parametrize("name", GC.CASES)
def test_oracle_matches_reference_cuda(name):
    path = os.path.join(HERE, "golden", "ref_%s.npz" % name)
    if not os.path.exists(path):
        pytest.skip("fixture %s not generated yet (tests/golden/make_golden.py on a GPU)" % os.path.basename(path))
    ref = np.load(path)
    geo, ang, img = GC.make(name)
    for k in GC.keys(name):
        tmax, tl2 = TOLS[k]
        got = _oracle_output(k, img, geo, ang, ref)
        want = ref[k]
        if k == "siddon":
            bad = _defect_mask(name, want.shape)
            off = np.abs(got - want) > tmax * np.abs(want).max()
            assert not (off & ~bad).any(), (name, np.argwhere(off & ~bad)[:5])
            got, want = got[~bad], want[~bad]
        mx, l2 = rel_err(got, want)
        assert mx <= tmax and l2 <= tl2, (name, k, mx, l2)


def _fine_line_integral(img, alpha, v, u, geo, n=400000):
    """Line integral of the voxelised image along one cone-beam ray by midpoint sampling (no
    Siddon traversal): axial geometry without offsets, source at (DSO, 0, 0) rotated by alpha
    about z, detector pixel (u, v) at x = -(DSD - DSO), u along +y, v along +z, both from the
    detector's lower corner, volume centred at the origin."""
    nz, ny, nx = img.shape
    dv, du = float(geo.dDetector[0]), float(geo.dDetector[1])
    nv, nu = int(geo.nDetector[0]), int(geo.nDetector[1])
    vox = np.asarray(geo.dVoxel, dtype=np.float64)[::-1]          # (x, y, z) mm
    s = np.array([geo.DSO, 0.0, 0.0])
    p = np.array([-(geo.DSD - geo.DSO), -nu * du / 2 + du / 2 + u * du, -nv * dv / 2 + dv / 2 + v * dv])
    c, sn = np.cos(alpha), np.sin(alpha)
    rot = np.array([[c, -sn, 0.0], [sn, c, 0.0], [0.0, 0.0, 1.0]])
    s, p = rot @ s, rot @ p
    t = (np.arange(n) + 0.5) / n
    pts = (s[None] + t[:, None] * (p - s)[None]) / vox + np.array([nx, ny, nz]) / 2.0
    idx = np.floor(pts).astype(np.int64)
    ok = np.all((idx >= 0) & (idx < np.array([nx, ny, nz])), axis=1)
    vals = np.zeros(n)
    vals[ok] = img[idx[ok, 2], idx[ok, 1], idx[ok, 0]]
    return float(vals.sum() * np.linalg.norm(p - s) / n)


def test_oracle_siddon_matches_fine_sampling_where_the_reference_errs():
    """On the rays where the reference's Siddon disagrees with the oracle, a midpoint-sampled
    line integral (4e5 samples per ray, independent of both traversals) sides with the oracle;
    on ordinary rays of the same view all three agree."""
    geo, ang, img = GC.make("c1")
    ref = np.load(os.path.join(HERE, "golden", "ref_c1.npz"))["siddon"]
    orc = O.ax(img, geo, ang, "Siddon")
    top = float(np.abs(orc).max())
    for view, col in REFERENCE_SIDDON_DEFECTS["c1"]:
        for v in (2, 16, 70, 101):
            fine = _fine_line_integral(img, float(ang[view]), v, col, geo)
            assert abs(fine - orc[view, v, col]) <= 2e-4 * top, (v, fine, orc[view, v, col])
            assert abs(fine - ref[view, v, col]) > 5e-3 * top, (v, fine, ref[view, v, col])
        for v, u in ((40, 30), (90, 100)):
            fine = _fine_line_integral(img, float(ang[view]), v, u, geo)
            assert abs(fine - orc[view, v, u]) <= 2e-4 * top and abs(fine - ref[view, v, u]) <= 5e-4 * top


def test_awtv_oracle_reduces_to_pocs_tv():
    """With a delta far above every difference all AwTV weights are 1: aw_pocs_tv is pocs_tv
    (the two drivers are the same code apart from the weights, GD_AwTV.cu:276 / GD_TV.cu:255)."""
    _, _, img = GC.make("small")
    a = O.aw_pocs_tv(img, GC.TV_ALPHA, GC.TV_ITERS, 1e12)
    t = O.pocs_tv(img, GC.TV_ALPHA, GC.TV_ITERS)
    mx, l2 = rel_err(a, t)
    assert mx <= 1e-6 and l2 <= 1e-7, (mx, l2)


def test_piccs_oracle_with_ratio_zero_is_bare_image_tv():
    """ratio = 0 drops the prior: PICCS is then a TV descent on the bare image, which differs
    from pocs_tv only at the first and last slices (no zero halo in z)."""
    _, _, img = GC.make("small")
    p0 = O.piccs_tv(img, np.zeros_like(img), GC.TV_ALPHA, 0.0, 1)
    p1 = O.piccs_tv(img, img * 0.5, GC.TV_ALPHA, 0.0, 1)
    assert np.array_equal(p0, p1)
    t = O.pocs_tv(img, GC.TV_ALPHA, 1)
    # interior slices step in the same direction; the scale differs through the global norm
    d_p, d_t = (p0 - img)[2:-2], (t - img)[2:-2]
    cos = float((d_p * d_t).sum() / np.sqrt((d_p * d_p).sum() * (d_t * d_t).sum()))
    assert cos > 0.99, cos


def _parker_case(name):
    from tests.golden.make_parker_golden import CASES, angles_for
    from tigre_b200.utilities.geometry import cone_geometry
    _, n, d, dsd, views, extra, q = next(c for c in CASES if c[0] == name)
    geo = cone_geometry((16, 16, 16), (16.0,) * 3, (n, n), (d, d), DSO=0.6 * dsd, DSD=dsd)
    return geo, angles_for(n, d, dsd, views, extra), q


@pytest.mark.parametrize("name", ["short_scan", "overscan", "q_half"])
def test_parker_oracle_matches_reference_weights(name):
    """FP64 Parker weights of the oracle against the reference's parkerweight.py outputs."""
    geo, ang, q = _parker_case(name)
    ref = np.load(os.path.join(HERE, "golden", "ref_parker.npz"))[name]
    got = O.parker_weights(geo, ang, q)
    assert got.shape == ref.shape
    np.testing.assert_allclose(got, ref, rtol=0, atol=1e-12)


@pytest.mark.parametrize("name", ["short_scan", "overscan", "q_half"])
def test_product_parker_weights_match_reference_weights(name):
    """The package's host-side Parker weights (float32) against the same reference outputs."""
    from tigre_b200.utilities import filtering as F
    geo, ang, q = _parker_case(name)
    ref = np.load(os.path.join(HERE, "golden", "ref_parker.npz"))[name]
    np.testing.assert_allclose(F.parker_weights(geo, ang, q), ref, rtol=0, atol=2e-7)


def test_parker_weights_follow_u_on_a_wide_detector():
    """On a non-square detector the weights vary along u with the u extent's fan angle
    (MATLAB/Utilities/ParkerWeight.m:17-20): a column at u and its mirror image swap their
    roles between the start and the end of the scan (beta -> span - beta)."""
    from tigre_b200.utilities.geometry import cone_geometry
    geo = cone_geometry((16, 16, 16), (16.0,) * 3, (20, 96), (0.8, 0.8), DSO=1000.0, DSD=1536.0)
    delta = np.arctan(0.5 * 96 * 0.8 / 1536.0)
    ang = np.linspace(0, np.pi + 2 * delta, 121).astype(np.float32)
    w = O.parker_weights(geo, ang)
    assert w.shape == (121, 96)
    np.testing.assert_allclose(w[:, ::-1], w[::-1, :], atol=1e-5)
    assert w.min() >= 0.0 and w.max() <= 1.0
    # every ray is weighted once over the short scan: opposite rays sum to one in the interior
    from tigre_b200.utilities import filtering as F
    np.testing.assert_allclose(F.parker_weights(geo, ang), w, atol=2e-7)


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_measure_quality_matches_reference(seed):
    """tigre_b200.utilities.Measure_Quality against the reference's own outputs."""
    from tests.golden.make_quality_golden import OPTS, pair
    from tigre_b200.utilities.Measure_Quality import Measure_Quality
    ref = np.load(os.path.join(HERE, "golden", "ref_quality.npz"))["seed%d" % seed]
    a, b = pair(seed)
    got = Measure_Quality(a, b, OPTS)
    np.testing.assert_allclose(got, ref, rtol=1e-6, atol=1e-12)
    for i, q in enumerate(OPTS):
        np.testing.assert_allclose(Measure_Quality(a, b, q), ref[i], rtol=1e-6, atol=1e-12)
