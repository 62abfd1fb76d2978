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


@pytest.mark.parametrize("name", GC.CASES)
def test_oracle_matches_reference_cuda(name):
    path = os.path.join(HERE, "golden", "ref_%s.npz" % name)
    ref = np.load(path)
    geo, ang, img = GC.make(name)
    got = {
        "siddon": O.ax(img, geo, ang, "Siddon"),
        "interpolated": O.ax(img, geo, ang, "interpolated"),
        "fdk": O.atb(ref["siddon"], geo, ang, "FDK"),
        "matched": O.atb(ref["siddon"], geo, ang, "matched"),
        "pocs_tv": O.pocs_tv(img, GC.TV_ALPHA, GC.TV_ITERS),
        "tvdenoise": O.tvdenoise((img - img.min()) / (img - img.min()).max(), GC.DENOISE_ITERS, GC.DENOISE_LAMBDA),
        "awtv": O.aw_pocs_tv(img, GC.TV_ALPHA, GC.TV_ITERS, GC.AWTV_DELTA),
        "piccs": O.piccs_tv(img, GC.piccs_prior(img), GC.TV_ALPHA, GC.PICCS_RATIO, GC.TV_ITERS),
    }
    for k, (tmax, tl2) in TOLS.items():
        mx, l2 = rel_err(got[k], ref[k])
        assert mx <= tmax and l2 <= tl2, (name, k, mx, l2)


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
