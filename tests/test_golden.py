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
    }
    for k, (tmax, tl2) in TOLS.items():
        mx, l2 = rel_err(got[k], ref[k])
        assert mx <= tmax and l2 <= tl2, (name, k, mx, l2)
