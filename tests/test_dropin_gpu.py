"""TIGRE's own Python package, unmodified, running on libtigre_b200.so.

tests/dropin/build.py compiles the reference's eight Cython extensions (_Ax, _Atb, _minTV,
_AwminTV, _minPICCS, _tv_proximal, _gpuUtils, _RandomNumberGenerator) from its own .pyx files
with the projector and regulariser CUDA sources replaced by this library, and puts them beside
a copy of the reference's Python package.  Here that package is imported as `tigre` and its
public calls -- tigre.Ax, tigre.Atb, minTV, tigre.algorithms.cgls -- are checked against the
FP64 oracle (bar 1e-5 relative for single operators; CGLS, whose vector algebra the reference
does in float32 numpy, 2e-4 on the iterate).
"""
import os

import numpy as np
import pytest

from tests import geometries as G
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-5
HERE = os.path.dirname(os.path.abspath(__file__))
DROPIN = os.path.join(HERE, "dropin", "_build")


@pytest.fixture(scope="module")
def T():
    from oracle import reference_package as RP
    if not RP.available("ours"):
        pytest.skip("drop-in build absent (tests/dropin/build.py needs the TIGRE source tree)")
    return RP.load("ours")


def _ref_geometry(T, ours):
    from oracle import reference_package as RP
    return RP.geometry_like(T, ours)


def _maps():
    with open("/proc/self/maps") as f:
        return f.read()


def test_reference_extensions_bind_this_library(T):
    import _Ax
    import _Atb
    import _minTV
    for m in (_Ax, _Atb, _minTV):
        assert os.path.dirname(m.__file__) == DROPIN, m.__file__
    maps = _maps()
    assert "tigre_b200/libtigre_b200.so" in maps
    assert "libref_" not in maps          # the reference's own CUDA build is not in this process


@pytest.mark.parametrize("ptype", ["Siddon", "interpolated"])
def test_reference_ax_matches_oracle(T, ptype):
    ours = G.odd_geometry()
    ang = G.angles(37, full=np.pi * 1.3)
    img = G.phantom(tuple(int(v) for v in ours.nVoxel), seed=1)
    got = T.Ax(img, _ref_geometry(T, ours), ang, ptype)
    mx, l2 = G.rel_err(got, O.ax(img, ours, ang, ptype))
    assert mx <= TOL and l2 <= TOL, (ptype, mx, l2)


@pytest.mark.parametrize("btype", ["FDK", "matched"])
def test_reference_atb_matches_oracle(T, btype):
    ours = G.c1_geometry()
    ang = G.angles(100)
    img = G.phantom((64, 64, 64), seed=0)
    proj = O.ax(img, ours, ang, "Siddon")
    got = T.Atb(proj, _ref_geometry(T, ours), ang, btype)
    mx, l2 = G.rel_err(got, O.atb(proj, ours, ang, btype))
    assert mx <= TOL and l2 <= TOL, (btype, mx, l2)


def test_reference_mintv_matches_oracle(T):
    from _minTV import minTV
    img = G.phantom((40, 48, 56), seed=7) + np.random.default_rng(7).normal(0, 0.002, (40, 48, 56))
    img = img.astype(np.float32)
    got = minTV(img, 0.002, 10)
    mx, l2 = G.rel_err(got, O.pocs_tv(img, 0.002, 10))
    assert mx <= TOL and l2 <= TOL, (mx, l2)


def test_reference_cgls_on_this_library_matches_oracle(T):
    """tigre.algorithms.cgls (krylov_subspace_algorithms.py:22-99), the reference's own driver,
    10 iterations at the small plain-method configuration (64^3, 128^2 @ 0.8 mm, 100 views)."""
    ours = G.c1_geometry()
    ang = G.angles(100)
    img = G.phantom((64, 64, 64), seed=0)
    proj = O.ax(img, ours, ang, "Siddon")
    x = T.algorithms.cgls(proj, _ref_geometry(T, ours), ang, 10)
    xr, _ = O.cgls(proj, ours, ang, 10)
    mx, l2 = G.rel_err(x, xr)
    print("reference cgls over libtigre_b200 vs FP64 oracle CGLS: max %.2e, L2 %.2e" % (mx, l2))
    assert l2 <= 2e-4, (mx, l2)
