"""Host entry points with volumes of 32 MiB or more move them through pinned bounce buffers
(api.cu: staged_h2d / staged_d2h).  The staged copies must give the same bytes as the driver's
pageable path: a 288 x 256 x 256 FP32 volume (72 MiB: one full 64 MiB chunk and a tail) through
the TV, noise and projector host calls, staging on (default) and off (TIGRE_OPT_HOST_STAGING = 0)."""
import numpy as np
import pytest

from tests import geometries as G

pytestmark = pytest.mark.gpu

SHAPE = (288, 256, 256)


def _volume():
    rng = np.random.default_rng(11)
    return (G.phantom(SHAPE, seed=2) + rng.normal(0, 1e-3, SHAPE)).astype(np.float32)


def _both(fn):
    from tigre_b200 import _native as N
    with N.option(N.OPT_HOST_STAGING, 0):
        direct = fn()
    staged = fn()
    return direct, staged


def test_staged_tv_round_trip_matches_direct():
    from tigre_b200.utilities.minTV import minTV
    img = _volume()
    direct, staged = _both(lambda: minTV(img, 0.002, 2))
    np.testing.assert_array_equal(staged, direct)
    assert not np.array_equal(staged, img)


def test_staged_noise_round_trip_matches_direct():
    from tigre_b200.utilities import CTnoise
    proj = np.abs(_volume()) * 4.0
    direct, staged = _both(lambda: CTnoise.add(proj, Poisson=1e5, Gaussian=np.array([0, 0.5]), seed=3))
    np.testing.assert_array_equal(staged, direct)


def test_staged_volume_upload_matches_device_path():
    import torch
    import tigre_b200 as tigre
    from tigre_b200.utilities.geometry import cone_geometry
    img = _volume()
    geo = cone_geometry(SHAPE, (float(SHAPE[0]), 256.0, 256.0), (64, 96), (4.0, 4.0))
    ang = G.angles(6)
    direct, staged = _both(lambda: tigre.Ax(img, geo, ang, "Siddon"))
    np.testing.assert_array_equal(staged, direct)
    dev = tigre.Ax(torch.from_numpy(img).cuda(), geo, ang, "Siddon").cpu().numpy()
    np.testing.assert_array_equal(staged, dev)
