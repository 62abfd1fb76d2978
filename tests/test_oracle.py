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


def test_rounding_oracle_nearest_bf16_matches_torch():
    import torch
    from oracle import rounding as R
    v = (np.random.default_rng(0).standard_normal(50000) * 1e3).astype(np.float32)
    v[:4] = [np.inf, -np.inf, 0.0, 1e-40]
    want = torch.from_numpy(v).bfloat16().float().numpy()
    np.testing.assert_array_equal(R.bf16_to_f32(R.bf16_bits_nearest(v)), want)


@pytest.mark.parametrize("dtype", ["bfloat16", "float16"])
def test_rounding_oracle_stochastic_picks_a_neighbour_without_bias(dtype):
    from oracle import rounding as R
    rng = np.random.default_rng(1)
    v = rng.uniform(0.5, 4.0, (64, 1000)).astype(np.float32)
    outs = np.stack([R.sart_update(v, np.zeros_like(v), np.ones(1000, np.float32), 1.0, False, dtype,
                                   "stochastic", seed=3, step=k) for k in range(200)])
    if dtype == "bfloat16":
        lo = R.bf16_to_f32(((v.view(np.uint32) >> 16) << 16).astype(np.uint32) >> 16)
        hi = R.bf16_to_f32((v.view(np.uint32) >> 16) + 1)
    else:
        h = v.astype(np.float16)
        lo = np.where(h.astype(np.float32) > v, np.nextafter(h, np.float16(-np.inf)), h).astype(np.float32)
        hi = np.where(h.astype(np.float32) < v, np.nextafter(h, np.float16(np.inf)), h).astype(np.float32)
    exact = lo == v
    assert np.all((outs == lo) | (outs == hi))
    assert np.all(outs[:, exact] == v[exact])
    # mean over 200 draws x 64000 values: unbiased to a few sigma of the pooled mean
    d = (outs.astype(np.float64) - v).mean(0) / (hi - lo).astype(np.float64).clip(min=1e-30)
    assert abs(d[~exact].mean()) < 5 * 0.5 / np.sqrt(200 * (~exact).sum())


def test_rounding_oracle_random_bits_depend_on_step_and_seed():
    from oracle import rounding as R
    a = R.random16(3, 20, seed=1, step=0)
    assert a.shape == (3, 20) and a.max() < 65536
    assert not np.array_equal(a, R.random16(3, 20, seed=1, step=1))
    assert not np.array_equal(a, R.random16(3, 20, seed=2, step=0))
    # a plane of 16 voxels draws the same bits as the first 16 of a plane of 20 (groups of 8)
    np.testing.assert_array_equal(a[0, :16], R.random16(1, 16, seed=1, step=0)[0])


def test_oracle_ossart_reduces_error_and_keeps_nonnegativity():
    geo = cone_geometry((16, 16, 16), (16.0,) * 3, (24, 32), (0.8, 0.8))
    ang = G.angles(12)
    img = G.phantom((16, 16, 16), seed=2)
    proj = O.ax(img, geo, ang, "Siddon")
    index = [np.arange(0, 6), np.arange(6, 12)]
    errs = []
    x = O.ossart(proj, geo, ang, 3, index, callback=lambda it, x: errs.append(np.linalg.norm(x - img)))
    assert x.min() >= 0 and errs[0] < np.linalg.norm(img) and errs[-1] < errs[0]
