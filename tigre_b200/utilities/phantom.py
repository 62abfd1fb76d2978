"""Seeded synthetic inputs: random-ellipsoid phantoms and Poisson noise.

Phantom: sum of `n` ellipsoids drawn from numpy.random.default_rng(seed):
centres uniform in +-0.6 of the half-extent, semi-axes uniform in
[0.05, 0.4] of the extent, ZYZ Euler angles uniform, additive attenuation
uniform in [0.002, 0.02] /mm, summed then clipped to [0, 0.02].  Voxel
centres sit on linspace(-1, 1, n) per axis and a voxel belongs to an
ellipsoid when its centre does -- the rasterisation rule of
Python/tigre/utilities/sl3d.py:60-121.

Noise: N ~ Poisson(I0 exp(-p)), p_noisy = -ln(max(N, 1) / I0).
"""
from __future__ import annotations

import numpy as np


def ellipsoid_params(n=10, seed=0):
    rng = np.random.default_rng(seed)
    centres = rng.uniform(-0.6, 0.6, size=(n, 3))          # (z, y, x), normalised
    axes = rng.uniform(0.05, 0.4, size=(n, 3)) * 2.0        # of the extent (2 in normalised units)
    eul = rng.uniform(0.0, 2.0 * np.pi, size=(n, 3))
    att = rng.uniform(0.002, 0.02, size=n)
    return centres, axes, eul, att


def _rot_zyz(a, b, c):
    ca, sa, cb, sb, cc, sc = np.cos(a), np.sin(a), np.cos(b), np.sin(b), np.cos(c), np.sin(c)
    rz1 = np.array([[ca, -sa, 0], [sa, ca, 0], [0, 0, 1]])
    ry = np.array([[cb, 0, sb], [0, 1, 0], [-sb, 0, cb]])
    rz2 = np.array([[cc, -sc, 0], [sc, cc, 0], [0, 0, 1]])
    return rz1 @ ry @ rz2


def random_ellipsoids(shape, n=10, seed=0, device=None, dtype=None):
    """Phantom of shape (nZ, nY, nX).  Returns numpy float32 when device is None,
    else a torch tensor on `device` (generated there, chunked over z)."""
    nz, ny, nx = (int(s) for s in shape)
    centres, axes, eul, att = ellipsoid_params(n, seed)
    if device is None:
        import torch
        out = random_ellipsoids(shape, n, seed, device="cpu")
        return out.numpy()
    import torch
    dev = torch.device(device)
    out = torch.zeros((nz, ny, nx), dtype=torch.float32, device=dev)
    zs = torch.linspace(-1, 1, nz, dtype=torch.float64, device=dev)
    ys = torch.linspace(-1, 1, ny, dtype=torch.float64, device=dev)
    xs = torch.linspace(-1, 1, nx, dtype=torch.float64, device=dev)
    step = max(1, int(2 ** 24 // max(1, nx * ny)))
    for e in range(n):
        R = torch.tensor(_rot_zyz(*eul[e]).T, dtype=torch.float64, device=dev)   # world -> body, (x,y,z) order
        cz, cy, cx = centres[e]
        az, ay, axx = axes[e]
        for z0 in range(0, nz, step):
            z1 = min(nz, z0 + step)
            Z, Y, X = torch.meshgrid(zs[z0:z1] - cz, ys - cy, xs - cx, indexing="ij")
            bx = R[0, 0] * X + R[0, 1] * Y + R[0, 2] * Z
            by = R[1, 0] * X + R[1, 1] * Y + R[1, 2] * Z
            bz = R[2, 0] * X + R[2, 1] * Y + R[2, 2] * Z
            inside = (bx / axx) ** 2 + (by / ay) ** 2 + (bz / az) ** 2 <= 1.0
            out[z0:z1] += inside.to(torch.float32) * float(att[e])
    out.clamp_(0.0, 0.02)
    if dtype is not None:
        out = out.to(dtype)
    return out


def poisson_noise(proj, I0=1e5, seed=0):
    """Poisson noise on line integrals (numpy or torch, same type back)."""
    if type(proj).__module__.startswith("torch"):
        import torch
        g = torch.Generator(device=proj.device)
        g.manual_seed(int(seed))
        lam = float(I0) * torch.exp(-proj.double())
        cnt = torch.poisson(lam, generator=g).clamp_(min=1.0)
        return (-torch.log(cnt / float(I0))).to(proj.dtype)
    rng = np.random.default_rng(seed)
    cnt = np.maximum(rng.poisson(float(I0) * np.exp(-proj.astype(np.float64))), 1.0)
    return (-np.log(cnt / float(I0))).astype(proj.dtype)
