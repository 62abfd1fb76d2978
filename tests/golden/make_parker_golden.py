"""Generate tests/golden/ref_parker.npz from the reference's own Parker weights.

    python tests/golden/make_parker_golden.py [TIGRE_ROOT]     # CPU only; default /root/reference

Python/tigre/utilities/parkerweight.py is plain numpy, so it is loaded straight from the TIGRE
source tree (not copied) and run on a stack of ones; the stored array is the weight it gives
each (view, detector column).  It is called on (nangles, nV, nU) stacks directly, i.e. with its
own formula, not through the reference's filtering.py, which transposes the stack first and so
applies the weights along v (its "TODO: Fix parker", filtering.py:14).  The cases use square
detectors and increasing angles, where the Python function and MATLAB/Utilities/ParkerWeight.m
(u axis, negated fan angle for increasing angles) coincide.
"""
import importlib.util
import os
import sys
import types
import warnings

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

# (name, detector pixels per side, pixel mm, DSD, views, span beyond pi + 2 * half fan angle of the
# detector edge (rad), q)
CASES = [
    ("short_scan", 64, 0.8, 1536.0, 90, 0.0, 1.0),        # the detector-edge fan angle: small overscan
    ("overscan", 48, 1.2, 1000.0, 61, 0.05, 1.0),       # wider overscan epsilon
    ("q_half", 40, 1.0, 800.0, 45, 0.02, 0.5),          # Wesarg's q < 1
]


def angles_for(n_det, d_det, dsd, views, extra):
    """Short-scan views over [0, pi + 2 delta_edge + extra], end angle included, with
    delta_edge = atan(n_det * d_det / 2 / dsd), the half fan angle to the detector's outer edge."""
    delta_edge = np.arctan(0.5 * n_det * d_det / dsd)
    return np.linspace(0.0, np.pi + 2 * delta_edge + extra, views).astype(np.float32)


def main():
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("TIGRE_REFERENCE", "/root/reference")
    path = os.path.join(root, "Python", "tigre", "utilities", "parkerweight.py")
    spec = importlib.util.spec_from_file_location("ref_parkerweight", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    out = {}
    for name, n, d, dsd, views, extra, q in CASES:
        geo = types.SimpleNamespace(sDetector=np.array([n * d, n * d]), dDetector=np.array([d, d]),
                                    DSD=np.full(views, dsd))
        ang = angles_for(n, d, dsd, views, extra)
        with warnings.catch_warnings():
            warnings.simplefilter("error")      # the cases are proper short scans: no warning expected
            w = mod.parkerweight(np.ones((views, n, n)), geo, ang.astype(np.float64), q)
        assert np.allclose(w, w[:, :1, :]), "weights must vary along u only"
        out[name] = w[:, 0, :].astype(np.float64)
        print(name, out[name].shape, float(out[name].min()), float(out[name].max()))
    np.savez_compressed(os.path.join(HERE, "ref_parker.npz"), **out)


if __name__ == "__main__":
    main()
