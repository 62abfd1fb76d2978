"""SART volume-update kernel and the storage precision of OS-SART, against the oracles.

* tigre_sart_update is bit-exact against the rounding oracle (oracle/rounding.py) for FP32,
  BF16 and FP16 storage, nearest and stochastic rounding, on the 16-byte path (nyx % 8 == 0)
  and the element path;
* stochastic rounding keeps updates below half a unit in the last place in expectation;
* OS-SART per iteration against the FP64 oracle OS-SART (oracle.ossart): FP32 storage within
  1e-4 relative, and the stated error of each 16-bit storage mode.
"""
import numpy as np
import pytest

from tests import geometries as G
from oracle import oracle as O
from oracle import rounding as R

pytestmark = pytest.mark.gpu

SHAPES = [(5, 16, 24), (3, 7, 9)]


def _inputs(shape, seed):
    rng = np.random.default_rng(seed)
    x = rng.uniform(-0.2, 1.0, shape).astype(np.float32)
    bp = (rng.standard_normal(shape) * 0.05).astype(np.float32)
    v = rng.uniform(0.5, 3.0, shape[1:]).astype(np.float32)
    v[0, 0] = np.inf            # set_v marks zero weights with inf
    bp[0, 0, 1] = -5.0          # a clipped voxel
    return x, bp, v


@pytest.mark.parametrize("noneg", [True, False])
@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("rounding", ["nearest", "stochastic"])
@pytest.mark.parametrize("dtype", ["float32", "bfloat16", "float16"])
def test_sart_update_bit_exact(dtype, rounding, shape, noneg):
    import torch
    from tigre_b200 import projectors as P
    x, bp, v = _inputs(shape, 1)
    xs = torch.from_numpy(x).cuda().to(getattr(torch, dtype))
    start = xs.float().cpu().numpy()
    P.sart_update_(xs, torch.from_numpy(bp).cuda(), torch.from_numpy(v).cuda(), 0.9, noneg, rounding,
                   seed=1234, step=7)
    want = R.sart_update(start, bp, v, 0.9, noneg, dtype, rounding, seed=1234, step=7)
    np.testing.assert_array_equal(xs.float().cpu().numpy(), want)


@pytest.mark.parametrize("dtype", ["bfloat16", "float16"])
def test_stochastic_rounding_stays_finite_near_the_largest_value(dtype):
    """Values just below the largest finite 16-bit number, pushed up by an update, stay finite
    under stochastic rounding (both storage types saturate like nearest rounding does not)."""
    import torch
    from tigre_b200 import projectors as P
    top = float(torch.finfo(getattr(torch, dtype)).max)
    x = np.full((2, 8, 16), top, np.float32)
    x[1] *= -1.0
    bp = np.zeros_like(x)
    bp[0] = top * 2 ** -9        # below one ulp of the largest value: rounds up or stays
    bp[1] = -top * 2 ** -9
    v = np.ones((8, 16), np.float32)
    xs = torch.from_numpy(x).cuda().to(getattr(torch, dtype))
    for step in range(4):
        P.sart_update_(xs, torch.from_numpy(bp).cuda(), torch.from_numpy(v).cuda(), 1.0, False, "stochastic",
                       seed=3, step=step)
    got = xs.float().cpu().numpy()
    assert np.isfinite(got).all()
    want = R.sart_update(x, bp, v, 1.0, False, dtype, "stochastic", seed=3, step=0)
    assert np.isfinite(want).all()


def test_sart_update_matches_reference_expression_fp32():
    """FP32: the fused kernel equals res + lmbda * 1.0 / V * bp followed by clip(min=0), evaluated
    as numpy evaluates it (iterative_recon_alg.py:389-401, :344-345)."""
    import torch
    from tigre_b200 import projectors as P
    x, bp, v = _inputs((4, 32, 40), 2)
    want = (x + np.float32(0.7) * np.float32(1.0) / v * bp).clip(min=0)
    xs = torch.from_numpy(x).cuda()
    P.sart_update_(xs, torch.from_numpy(bp).cuda(), torch.from_numpy(v).cuda(), 0.7)
    np.testing.assert_array_equal(xs.cpu().numpy(), want)


@pytest.mark.parametrize("dtype,delta", [("bfloat16", 1e-3), ("float16", 1e-4)])
def test_stochastic_rounding_keeps_small_updates(dtype, delta):
    """100 updates of delta below half an ulp of 1.0: nearest rounding drops all of them,
    stochastic rounding adds 100 delta in expectation (5-sigma bound on the mean)."""
    import torch
    from tigre_b200 import projectors as P
    shape = (16, 128, 128)
    T = getattr(torch, dtype)
    bp = torch.full(shape, delta, dtype=torch.float32, device="cuda")
    v = torch.ones(shape[1:], dtype=torch.float32, device="cuda")
    near = torch.ones(shape, dtype=T, device="cuda")
    sr = torch.ones(shape, dtype=T, device="cuda")
    steps = 100
    for k in range(steps):
        P.sart_update_(near, bp, v, 1.0, True, "nearest")
        P.sart_update_(sr, bp, v, 1.0, True, "stochastic", seed=99, step=k)
    assert float(near.float().max()) == 1.0 and float(near.float().min()) == 1.0
    vals = sr.double()
    mean = float(vals.mean())
    ulp = 2.0 ** -7 if dtype == "bfloat16" else 2.0 ** -10
    sigma = ulp * np.sqrt(steps / 4.0) / np.sqrt(vals.numel())
    assert abs(mean - (1.0 + steps * delta)) < 5 * sigma + 1e-12, (mean, 1.0 + steps * delta, sigma)


def test_sart_update_rejects_bad_arguments():
    import torch
    from tigre_b200 import projectors as P
    x = torch.zeros((2, 4, 8), device="cuda")
    with pytest.raises(ValueError):
        P.sart_update_(x, torch.zeros((2, 4, 8), device="cuda", dtype=torch.float16),
                       torch.ones((4, 8), device="cuda"), 1.0)
    with pytest.raises(ValueError):
        P.sart_update_(x, torch.zeros((2, 4, 8), device="cuda"), torch.ones((8, 4), device="cuda"), 1.0)


def _case(n=32, views=30, seed=3):
    from tigre_b200.utilities.geometry import cone_geometry
    geo = cone_geometry((n, n, n), (float(n),) * 3, (48, 64), (0.8, 0.8))
    return geo, G.angles(views), G.phantom((n, n, n), seed=seed)


# per-iteration relative L2 error bounds against the FP64 oracle after 5 iterations of
# OS-SART (30 views, blocksize 10, 32^3); FP32 is the parity bar, the 16-bit bounds state the
# storage error (measured values are printed with -s)
STORAGE_BOUNDS = {("float32", "nearest"): 1e-4,
                  ("bfloat16", "nearest"): 2e-2, ("bfloat16", "stochastic"): 2e-2,
                  ("float16", "nearest"): 3e-3, ("float16", "stochastic"): 3e-3}


@pytest.mark.parametrize("order", [None, "angularDistance"])
def test_ossart_per_iteration_vs_fp64_oracle(order):
    import torch
    import tigre_b200 as tigre
    from tigre_b200.utilities.order_subsets import order_subsets
    geo, ang, img = _case()
    proj = O.ax(img, geo, ang, "Siddon")
    ang3 = np.zeros((len(ang), 3), dtype=np.float32)
    ang3[:, 0] = ang
    _, index = order_subsets(ang3, 10, order)
    niter = 5
    ref = []
    O.ossart(proj, geo, ang, niter, index, callback=lambda it, x: ref.append(x.copy()))
    for (dtype, rounding), bound in STORAGE_BOUNDS.items():
        got = []
        st = None if dtype == "float32" else getattr(torch, dtype)
        tigre.algorithms.ossart(proj, geo, ang, niter, blocksize=10, OrderStrategy=order, storage=st,
                                rounding=rounding, seed=5,
                                callback=lambda it, x: got.append(x.double().cpu().numpy()))
        errs = [np.linalg.norm(g - r) / np.linalg.norm(r) for g, r in zip(got, ref)]
        print("%s %s %s per-iteration rel L2 vs FP64 oracle: %s" % (order, dtype, rounding,
                                                                     " ".join("%.2e" % e for e in errs)))
        assert len(errs) == niter and max(errs) <= bound, (dtype, rounding, errs)


def test_precision_configuration_scaled_per_iteration_vs_fp64_oracle():
    """The precision configuration (512^3 @ 0.5 mm, 1024 x 768 @ 0.4 mm, 720 views, 20 OS-SART
    iterations of 20 subsets) scaled by 1/4 per axis so that the FP64 oracle's whole trajectory
    is affordable on the host: 128^3 @ 2 mm (256 mm), 256 x 192 @ 1.6 mm, 180 views, blocksize 9
    (20 subsets), 20 iterations.  Per iteration, the relative L2 error of the FP32 path and of
    BF16 storage (nearest and stochastic rounding) against the FP64 oracle OS-SART."""
    import torch
    import tigre_b200 as tigre
    from tigre_b200.utilities.geometry import cone_geometry
    from tigre_b200.utilities.order_subsets import order_subsets
    geo = cone_geometry((128, 128, 128), (256.0, 256.0, 256.0), (192, 256), (1.6, 1.6), DSO=1000.0, DSD=1536.0)
    ang = np.linspace(0, 2 * np.pi, 180, endpoint=False).astype(np.float32)
    img = G.phantom((128, 128, 128), seed=0)
    proj = O.ax(img, geo, ang, "Siddon")
    ang3 = np.zeros((180, 3), dtype=np.float32)
    ang3[:, 0] = ang
    _, index = order_subsets(ang3, 9, None)
    niter = 20
    ref = []
    O.ossart(proj, geo, ang, niter, index, callback=lambda it, x: ref.append(x.copy()))
    bounds = {("float32", "nearest"): 1e-4, ("bfloat16", "nearest"): 3e-2, ("bfloat16", "stochastic"): 3e-2}
    for (dtype, rounding), bound in bounds.items():
        got = []
        st = None if dtype == "float32" else getattr(torch, dtype)
        tigre.algorithms.ossart(proj, geo, ang, niter, blocksize=9, storage=st, rounding=rounding, seed=5,
                                callback=lambda it, x: got.append(x.double().cpu().numpy()))
        errs = [np.linalg.norm(g - r) / np.linalg.norm(r) for g, r in zip(got, ref)]
        print("scaled precision configuration, %s %s, per-iteration rel L2 vs FP64 oracle: %s" % (
            dtype, rounding, " ".join("%.2e" % e for e in errs)))
        assert len(errs) == niter and max(errs) <= bound, (dtype, rounding, errs)
