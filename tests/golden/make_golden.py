"""Generate tests/golden/*.npz from the reference's own CUDA build (oracle/_ref) on a GPU.

    python tests/golden/make_golden.py       # needs a CUDA device and oracle/_ref built

Each fixture stores the case name, the seed and the reference's outputs for
Siddon and interpolated projection, FDK and matched backprojection (of the
reference's own Siddon projections), pocs_tv, tvdenoising, aw_pocs_tv and piccs_tv.  Inputs are regenerated
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
    # usage: make_golden.py [--keys k1,k2] [OUT_DIR [CASE ...]]   (default: this directory, every case)
    # --keys computes only those outputs and merges them into the fixtures already in OUT_DIR.
    args = sys.argv[1:]
    keys = None
    if args[:1] == ["--keys"]:
        keys = set(args[1].split(","))
        args = args[2:]
    out_dir = args[0] if args else os.path.dirname(os.path.abspath(__file__))
    names = args[1:] or GC.CASES
    os.makedirs(out_dir, exist_ok=True)
    for name in names:
        geo, ang, img = GC.make(name)
        path = os.path.join(out_dir, "ref_%s.npz" % name)
        if keys is not None:
            res = dict(np.load(path))
            _tv_family(res, img, keys)
            np.savez_compressed(path, **res)
            print(name, "updated", sorted(keys))
            continue
        res = {}
        want = set(GC.keys(name))
        res["siddon"], _ = ref.ax(img, geo, ang, "Siddon")
        res["interpolated"], _ = ref.ax(img, geo, ang, "interpolated")
        res["fdk"], _ = ref.atb(res["siddon"], geo, ang, "FDK")
        res["matched"], _ = ref.atb(res["siddon"], geo, ang, "matched")
        if "pocs_tv" in want:
            res["pocs_tv"], _ = ref.pocs_tv(img, GC.TV_ALPHA, GC.TV_ITERS)
        if "tvdenoise" in want:
            scaled = (img - img.min()) / (img - img.min()).max()
            res["tvdenoise"], _ = ref.tvdenoise(scaled.astype(np.float32), GC.DENOISE_LAMBDA, GC.DENOISE_ITERS)
        _tv_family(res, img, want & {"awtv", "piccs"})
        np.savez_compressed(path, **res)
        print(name, {k: v.shape for k, v in res.items()})


def _tv_family(res, img, keys):
    """AwminTV and minPICCS outputs of the reference (aw_pocs_tv, piccs_tv)."""
    if "awtv" in keys:
        res["awtv"], _ = ref.aw_pocs_tv(img, GC.TV_ALPHA, GC.TV_ITERS, GC.AWTV_DELTA)
    if "piccs" in keys:
        res["piccs"], _ = ref.piccs_tv(img, GC.piccs_prior(img), GC.TV_ALPHA, GC.PICCS_RATIO, GC.TV_ITERS)


if __name__ == "__main__":
    main()
