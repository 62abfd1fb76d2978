"""Geometries and inputs shared by the parity tests (seeded, small enough for the oracle)."""
import numpy as np

from tigre_b200.utilities.geometry import cone_geometry
from tigre_b200.utilities.phantom import random_ellipsoids


def c1_geometry():
    """64^3 @ 1 mm, DSO 1000, DSD 1536, 128x128 @ 0.8 mm (the small plain-method case)."""
    return cone_geometry((64, 64, 64), (64.0, 64.0, 64.0), (128, 128), (0.8, 0.8))


def odd_geometry():
    """Odd, anisotropic sizes with offsets: exercises tails and every axis of the frames."""
    g = cone_geometry((61, 67, 73), (61 * 0.9, 67 * 1.1, 73 * 1.0), (97, 131), (0.9, 0.7))
    g.offOrigin = np.array((1.5, -2.0, 3.25))
    g.offDetector = np.array((2.4, -1.6))
    g.COR = 0.7
    return g


def tilted_geometry():
    """Detector roll/pitch/yaw and non-axial Euler angles (theta, psi != 0)."""
    g = cone_geometry((48, 40, 44), (48.0, 40.0, 44.0), (72, 88), (0.8, 0.8))
    g.rotDetector = np.array((0.03, -0.02, 0.05))
    return g


def steep_geometry():
    """Short source distance and 0.25 mm slices: rays climb up to ~1.5 slices per xy cell,
    so the column projector takes its several-crossings-per-cell path."""
    return cone_geometry((40, 48, 48), (10.0, 48.0, 48.0), (128, 96), (1.5, 1.5), DSO=150.0, DSD=250.0)


def angles(n, full=2 * np.pi, tilt=False, seed=3):
    a = np.linspace(0, full, n, endpoint=False).astype(np.float32)
    if not tilt:
        return a
    rng = np.random.default_rng(seed)
    out = np.zeros((n, 3), dtype=np.float32)
    out[:, 0] = a
    out[:, 1] = rng.uniform(-0.3, 0.3, n)
    out[:, 2] = rng.uniform(-0.3, 0.3, n)
    return out


def phantom(shape, seed=0):
    return random_ellipsoids(shape, n=10, seed=seed)


def rel_err(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    scale = max(np.abs(b).max(), 1e-30)
    return float(np.abs(a - b).max() / scale), float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))
