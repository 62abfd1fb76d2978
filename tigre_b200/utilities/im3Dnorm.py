"""Image norms, drop-in for Python/tigre/utilities/im3Dnorm.py:4-39."""
import numpy as np


def im3DNORM(img, normind, varargin=None):  # noqa: N802
    if type(img).__module__.startswith("torch"):
        img = img.detach().cpu().numpy()
    if normind in (np.inf, -np.inf, "fro", "nuc") or type(normind) is int:
        return np.linalg.norm(img.ravel(), normind)
    if normind == "TV":
        gx, gy, gz = np.diff(img, axis=2), np.diff(img, axis=1), np.diff(img, axis=0)
        gx, gy, gz = gx[:-1, :-1, :], gy[:-1, :, :-1], gz[:, :-1, :-1]
        return np.sum(np.sqrt(gx * gx + gy * gy + gz * gz))
    raise ValueError("norm not recognized: " + str(normind))
