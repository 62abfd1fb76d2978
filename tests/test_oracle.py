"""CPU tests of the FP64 oracle: pinned against analytic answers before it is trusted."""
import numpy as np
import pytest

from tests import geometries as G
from oracle import oracle as O
from tigre_b200.utilities.geometry import cone_geometry


def _chord_mm(S, P, lo, hi):
    d = P - S
    t0, t1 = -np.inf, np.inf
    for a in range(3):
        if abs(d[a]) < 1e-12:
            if S[a] < lo[a] or S[a] > hi[a]:
                return 0.0
            continue
        ta, tb = (lo[a] - S[a]) / d[a], (hi[a] - S[a]) / d[a]
        t0, t1 = max(t0, min(ta, tb)), min(t1, max(ta, tb))
    return max(t1 - t0, 0.0) * np.linalg.norm(d)


def _pixel_world(alpha, u, v, nu, nv, du, dv, dso, dsd, offu=0.0, offv=0.0):
    ca, sa = np.cos(alpha), np.sin(alpha)
    y = du * (u + 0.5 - nu / 2) + offu
    z = dv * (v + 0.5 - nv / 2) + offv
    x = -(dsd - dso)
    S = np.array([dso * ca, dso * sa, 0.0])
    P = np.array([x * ca - y * sa, x * sa + y * ca, z])
    return S, P


@pytest.mark.parametrize("off", [(0.0, 0.0, 0.0), (3.0, -5.0, 7.5)])
def test_siddon_uniform_volume_equals_chord(off):
    """Siddon of a constant volume = value x chord length through the box (pins the
    frames: rotation sense, detector flip, offsets, mm scaling)."""
    g = cone_geometry((40, 48, 56), (40 * 1.25, 48 * 1.0, 56 * 0.75), (60, 70), (1.1, 0.9))
    g.offOrigin = np.array(off)
    g.offDetector = np.array((1.3, -2.1))
    ang = np.array([0.0, 0.7, 2.2, 4.0], dtype=np.float32)
    img = np.full((40, 48, 56), 0.5, dtype=np.float32)
    p = O.ax(img, g, ang, "Siddon")
    half = np.array([56 * 0.75, 48 * 1.0, 40 * 1.25]) / 2
    centre = np.array([off[2], off[1], off[0]])
    errs = []
    for i, a in enumerate(ang.astype(np.float64)):
        for (u, v) in [(0, 0), (35, 30), (69, 59), (10, 50), (50, 5)]:
            S, P = _pixel_world(a, u, v, 70, 60, 0.9, 1.1, 1000.0, 1536.0, offu=-2.1, offv=1.3)
            c = _chord_mm(S, P, centre - half, centre + half) * 0.5
            errs.append(abs(c - p[i, v, u]) / max(abs(c), 1e-3))
    assert max(errs) < 2e-6


def test_interp_uniform_volume_close_to_chord():
    g = G.c1_geometry()
    ang = G.angles(5)
    img = np.ones((64, 64, 64), dtype=np.float32)
    pi = O.ax(img, g, ang, "interpolated")
    ps = O.ax(img, g, ang, "Siddon")
    # central rays cross the cube face-on: both equal the 64 mm chord
    assert abs(pi[0, 64, 64] - 64.0) < 1e-3 and abs(ps[0, 64, 64] - 64.0) < 1e-4
    # rays well inside the faces differ only by the half-voxel trilinear ramp at entry
    # and exit (rays that skim a face within half a voxel see a blurred face instead)
    core = np.zeros_like(ps, dtype=bool)
    core[:, 34:94, 34:94] = True
    assert np.abs(pi[core] - ps[core]).max() < 1.0


def test_matched_is_near_adjoint_of_siddon():
    g = G.c1_geometry()
    ang = G.angles(30)
    rng = np.random.default_rng(2)
    x = rng.random((64, 64, 64), dtype=np.float32)
    y = rng.random((30, 128, 128), dtype=np.float32)
    lhs = float((O.ax(x, g, ang, "Siddon").astype(np.float64) * y).sum())
    rhs = float((x.astype(np.float64) * O.atb(y, g, ang, "matched")).sum())
    assert abs(lhs - rhs) / abs(lhs) < 0.02


def test_fdk_weight_uniform_projection():
    """FDK backprojection of all-ones projections: each view adds (DSO/U)^2 inside the cone."""
    g = G.c1_geometry()
    ang = G.angles(1)
    proj = np.ones((1, 128, 128), dtype=np.float32)
    v = O.atb(proj, g, ang, "FDK")
    # voxel (x, y) at the centre has U = DSO -> weight 1
    assert abs(v[32, 32, 32] - 1.0) < 0.05
    # a voxel displaced toward the source (x > 0 at alpha=0) is magnified more: U < DSO -> weight > 1
    xw = -(64 - 1) * 0.5 + 60 * 1.0
    expected = (1000.0 / (1000.0 - xw)) ** 2
    assert abs(v[32, 32, 60] - expected) < 1e-4 * expected


def test_tv_gradient_matches_finite_differences_of_tv():
    rng = np.random.default_rng(0)
    x = rng.normal(0, 1, (5, 6, 7)).astype(np.float32)

    def tv(f):
        f = f.astype(np.float64)
        p = np.concatenate([np.zeros((1,) + f.shape[1:]), f, np.zeros((1,) + f.shape[1:])], axis=0)
        dz = p[1:] - p[:-1]                     # (nz+1) slices incl. the zero halo above
        dy = np.zeros_like(dz); dy[:-1, 1:, :] = f[:, 1:, :] - f[:, :-1, :]
        dx = np.zeros_like(dz); dx[:-1, :, 1:] = f[:, :, 1:] - f[:, :, :-1]
        return np.sqrt(dz ** 2 + dy ** 2 + dx ** 2).sum()

    g = O.tv_gradient(x)
    h = 1e-3
    for idx in [(0, 0, 0), (4, 5, 6), (2, 3, 3), (4, 0, 6)]:
        xp = x.astype(np.float64).copy(); xp[idx] += h
        xm = x.astype(np.float64).copy(); xm[idx] -= h
        fd = (tv(xp) - tv(xm)) / (2 * h)
        assert abs(fd - g[idx]) < 1e-3 * max(1, abs(fd)), (idx, fd, g[idx])


def test_pocs_tv_reduces_tv():
    img = G.phantom((16, 16, 16), seed=9) + np.random.default_rng(1).normal(0, 2e-3, (16, 16, 16)).astype(np.float32)
    out = O.pocs_tv(img, 0.01, 10)
    g0 = np.abs(np.diff(img, axis=0)).sum() + np.abs(np.diff(img, axis=1)).sum() + np.abs(np.diff(img, axis=2)).sum()
    g1 = np.abs(np.diff(out, axis=0)).sum() + np.abs(np.diff(out, axis=1)).sum() + np.abs(np.diff(out, axis=2)).sum()
    assert g1 < g0


def test_segment_counts_and_miss():
    g = G.c1_geometry()
    img = np.ones((64, 64, 64), dtype=np.float32)
    p, cnt = O.ax(img, g, G.angles(2), "Siddon", return_counts=True)
    assert cnt.max() > 64 and cnt.min() >= 0
    g.offOrigin = np.array((500.0, 0.0, 0.0))
    p2 = O.ax(img, g, G.angles(2), "Siddon")
    assert np.all(p2 == 0)
