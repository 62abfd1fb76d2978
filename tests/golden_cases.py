"""Small seeded cases whose reference outputs are stored in tests/golden/."""
import numpy as np

from tigre_b200.utilities.geometry import cone_geometry, geometry
from tigre_b200.utilities.phantom import random_ellipsoids

TV_ALPHA = 0.002
TV_ITERS = 10
DENOISE_LAMBDA = 15.0
DENOISE_ITERS = 30
AWTV_DELTA = -0.005       # AwminTV's default delta (_AwminTV.pyx:33)
PICCS_RATIO = 0.95        # minPICCS's default ratio (_minPICCS.pyx:39)


def piccs_prior(img):
    """Prior image of the PICCS fixtures: the image shifted by one voxel in x and y, scaled by 0.9."""
    return (0.9 * np.roll(np.roll(img, 1, axis=2), 1, axis=1)).astype(np.float32)


CASES = ("small", "offsets", "parallel", "rotated", "c1")

# outputs stored per case (default: every output); the C1-size case keeps the projector pair only
KEYS = {"c1": ("siddon", "interpolated", "fdk", "matched")}
ALL_KEYS = ("siddon", "interpolated", "fdk", "matched", "pocs_tv", "tvdenoise", "awtv", "piccs")


def keys(name):
    return KEYS.get(name, ALL_KEYS)


def make(name):
    if name == "small":
        geo = cone_geometry((32, 32, 32), (32.0, 32.0, 32.0), (48, 64), (0.8, 0.8))
        ang = np.linspace(0, 2 * np.pi, 12, endpoint=False).astype(np.float32)
        img = random_ellipsoids((32, 32, 32), seed=21)
    elif name == "offsets":
        geo = cone_geometry((24, 30, 28), (24 * 1.1, 30 * 0.9, 28.0), (40, 52), (0.9, 0.7))
        geo.offOrigin = np.array((1.0, -1.5, 2.0))
        geo.offDetector = np.array((1.2, -0.8))
        ang = np.linspace(0.1, 1.7 * np.pi, 10, endpoint=False).astype(np.float32)
        img = random_ellipsoids((24, 30, 28), seed=22)
    elif name == "parallel":
        # parallel beam with origin offsets, a horizontal detector offset and COR.  No vertical
        # detector offset: the reference's parallel Siddon keeps one z index per ray
        # (Siddon_projection_parallel.cu:224-266), so it is exact only for rays without a
        # z component, which a vertical offset would give (its source is not offset).
        geo = geometry(mode="parallel", nVoxel=np.array([20, 26, 30]))
        geo.offOrigin = np.array((0.5, -1.0, 1.5))
        geo.offDetector = np.array((0.0, 0.6))
        geo.COR = 0.3
        ang = np.linspace(0.05, np.pi, 9, endpoint=False).astype(np.float32)
        img = random_ellipsoids((20, 26, 30), seed=23)
    elif name == "rotated":
        # detector roll/pitch/yaw, non-axial Euler angles (theta, psi), centre-of-rotation shift
        # and origin/detector offsets: every term of the reference's geometry frames
        geo = cone_geometry((26, 30, 34), (26 * 1.1, 30.0, 34 * 0.9), (44, 56), (0.9, 0.8))
        geo.rotDetector = np.array((0.04, -0.03, 0.05))
        geo.COR = 0.6
        geo.offOrigin = np.array((0.8, 1.2, -1.0))
        geo.offDetector = np.array((-1.1, 0.9))
        rng = np.random.default_rng(24)
        ang = np.zeros((11, 3), dtype=np.float32)
        ang[:, 0] = np.linspace(0.2, 2 * np.pi, 11, endpoint=False)
        ang[:, 1] = rng.uniform(-0.25, 0.25, 11)
        ang[:, 2] = rng.uniform(-0.25, 0.25, 11)
        img = random_ellipsoids((26, 30, 34), seed=24)
    elif name == "c1":
        # the small plain-method configuration (64^3 @ 1 mm, 128 x 128 @ 0.8 mm, DSO 1000 /
        # DSD 1536), on 12 of its 100 views to keep the fixture small
        geo = cone_geometry((64, 64, 64), (64.0, 64.0, 64.0), (128, 128), (0.8, 0.8))
        ang = np.linspace(0, 2 * np.pi, 100, endpoint=False).astype(np.float32)[::9][:12]
        img = random_ellipsoids((64, 64, 64), seed=0)
    else:
        raise KeyError(name)
    return geo, ang, img.astype(np.float32)
