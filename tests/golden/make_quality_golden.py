"""Generate tests/golden/ref_quality.npz from the reference's Measure_Quality.

    python tests/golden/make_quality_golden.py [TIGRE_ROOT]      # CPU only; default /root/reference

Python/tigre/utilities/Measure_Quality.py is plain numpy: it is loaded from the TIGRE source tree
(not copied) and evaluated on seeded image pairs; the fixture stores the inputs' seeds and its
outputs for every measure.
"""
import importlib.util
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
OPTS = ["RMSE", "nRMSE", "CC", "MSSIM", "UQI", "SSD"]


def pair(seed):
    rng = np.random.default_rng(seed)
    a = rng.uniform(0.0, 1.0, (12, 10, 14)).astype(np.float32)
    b = (a + rng.normal(0.0, 0.1, a.shape)).astype(np.float32)
    return a, b


def main():
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("TIGRE_REFERENCE", "/root/reference")
    path = os.path.join(root, "Python", "tigre", "utilities", "Measure_Quality.py")
    spec = importlib.util.spec_from_file_location("ref_measure_quality", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    out = {}
    for seed in (1, 2, 3):
        a, b = pair(seed)
        out["seed%d" % seed] = np.asarray(mod.Measure_Quality(a, b, OPTS), dtype=np.float64)
    np.savez_compressed(os.path.join(HERE, "ref_quality.npz"), **out)
    print({k: v for k, v in out.items()})


if __name__ == "__main__":
    main()
