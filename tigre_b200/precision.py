"""Storage-precision study: OS-SART with BF16 (or FP16) volume and projection storage against the
same iteration in FP32, on the device.

    python -m tigre_b200.precision --size 512 --views 720 --iters 20 --blocksize 36 --out prec.json

Workload (the precision configuration): a seeded random-ellipsoid phantom of size^3 voxels over a
256 mm cube, cone beam DSO 1000 / DSD 1536, 1024 x 768 detector at 0.4 mm (scaled with size),
`views` angles over 2 pi, OS-SART with `views / blocksize` subsets per iteration (Siddon forward,
FDK-weighted backprojection, nonnegativity).  Both runs start from zero on the same FP32
projections; the 16-bit runs store the iterate and the projections in BF16 (or FP16) and
accumulate in FP32, once with round-to-nearest and once with stochastic rounding of the volume
updates; the "_vol" runs keep the projections in FP32 and store only the volume in 16 bits,
which separates the two sources of storage error.  Reported per iteration: the relative RMS difference of each 16-bit iterate from the FP32
one, each iterate's relative RMS error against the phantom, and the wall time per iteration.  The FP32 path
itself agrees with the FP64 oracle to 1e-5 per operator (the parity tests), so the BF16-FP32
difference is the storage error against the FP64 reference up to that bound.
"""
from __future__ import annotations

import json
import time

import numpy as np


def run(size=512, views=720, iters=20, blocksize=36, storage="bfloat16", seed=0, log=None):
    import torch
    from .algorithms.art import ossart
    from .utilities.geometry import cone_geometry
    from .utilities.phantom import random_ellipsoids
    from . import _native as N, projectors as P
    scale = size / 512.0
    nu, nv = int(round(1024 * scale)), int(round(768 * scale))
    geo = cone_geometry((size,) * 3, (256.0,) * 3, (nv, nu), (0.4 / scale, 0.4 / scale))
    ang = np.zeros((views, 3), dtype=np.float32)
    ang[:, 0] = np.linspace(0, 2 * np.pi, views, endpoint=False)
    img = random_ellipsoids((size,) * 3, seed=seed, device="cuda")
    plan = N.get_plan(N.checked_geometry(geo, ang), img.device.index)
    proj = P.ax(img, plan, "Siddon")
    inorm = float(img.double().norm())
    traces = {}
    st16 = getattr(torch, storage)
    modes = (("fp32", None, "nearest", None), (storage, st16, "nearest", None),
             (storage + "_sr", st16, "stochastic", None), (storage + "_vol", st16, "nearest", torch.float32),
             (storage + "_vol_sr", st16, "stochastic", torch.float32))
    for name, st, rounding, pst in modes:
        xs, ts = [], []
        t = [time.perf_counter()]

        def cb(it, x):
            torch.cuda.synchronize()
            ts.append(time.perf_counter() - t[0])
            xs.append(x.float().clone())
            t[0] = time.perf_counter()
        torch.cuda.synchronize()
        t[0] = time.perf_counter()
        ossart(proj, geo, ang, iters, blocksize=blocksize, storage=st, rounding=rounding, seed=seed + 1,
               proj_storage=pst, callback=cb, verbose=False)
        traces[name] = (xs, ts)
    rows = []
    for it in range(iters):
        a = traces["fp32"][0][it]
        an = float(a.double().norm())
        row = {"iter": it + 1}
        for name, _, _, _ in modes:
            b = traces[name][0][it]
            if name != "fp32":
                row["rel_rms_%s_vs_fp32" % name] = float((b - a).double().norm()) / max(an, 1e-30)
            row["rel_err_%s_vs_phantom" % name] = float((b - img).double().norm()) / inorm
            row["s_%s" % name] = traces[name][1][it]
        rows.append(row)
        if log:
            log(json.dumps(rows[-1]))
    return {"size": size, "views": views, "iters": iters, "blocksize": blocksize, "storage": storage,
            "rows": rows}


def main(argv=None):
    import argparse
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--size", type=int, default=512)
    ap.add_argument("--views", type=int, default=720)
    ap.add_argument("--iters", type=int, default=20)
    ap.add_argument("--blocksize", type=int, default=36)
    ap.add_argument("--storage", default="bfloat16", choices=["bfloat16", "float16"])
    ap.add_argument("--out", default=None)
    args = ap.parse_args(argv)
    res = run(args.size, args.views, args.iters, args.blocksize, args.storage, log=print)
    if args.out:
        json.dump(res, open(args.out, "w"), indent=1)


if __name__ == "__main__":
    main()
