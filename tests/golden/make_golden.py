"""Generate tests/golden/*.npz from the reference's own CUDA build (oracle/_ref) on a GPU.

    python tests/golden/make_golden.py       # needs a CUDA device and oracle/_ref built

Each fixture stores the case name, the seed and the reference's outputs for
Siddon and interpolated projection, FDK and matched backprojection (of the
reference's own Siddon projections) and pocs_tv.  Inputs are regenerated
from the seed by tests/geometries.py, so only outputs are stored.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import ref  # noqa: E402
from tests import golden_cases as GC  # noqa: E402


def main():
    # usage: make_golden.py [OUT_DIR [CASE ...]]   (default: this directory, every case)
    out_dir = sys.argv[1] if len(sys.argv) > 1 else os.path.dirname(os.path.abspath(__file__))
    names = sys.argv[2:] or GC.CASES
    os.makedirs(out_dir, exist_ok=True)
    for name in names:
        geo, ang, img = GC.make(name)
        res = {}
        res["siddon"], _ = ref.ax(img, geo, ang, "Siddon")
        res["interpolated"], _ = ref.ax(img, geo, ang, "interpolated")
        res["fdk"], _ = ref.atb(res["siddon"], geo, ang, "FDK")
        res["matched"], _ = ref.atb(res["siddon"], geo, ang, "matched")
        res["pocs_tv"], _ = ref.pocs_tv(img, GC.TV_ALPHA, GC.TV_ITERS)
        scaled = (img - img.min()) / (img - img.min()).max()
        res["tvdenoise"], _ = ref.tvdenoise(scaled.astype(np.float32), GC.DENOISE_LAMBDA, GC.DENOISE_ITERS)
        np.savez_compressed(os.path.join(out_dir, "ref_%s.npz" % name), **res)
        print(name, {k: v.shape for k, v in res.items()})


if __name__ == "__main__":
    main()
