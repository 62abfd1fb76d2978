#!/usr/bin/env python
"""Benchmark of the projector pair at 512^3 (one JSON line on rank 0).

Workload (the metric configuration): float32 512^3 volume @ 0.5 mm (256 mm),
random-ellipsoid phantom (seed = rank), cone beam DSO 1000 mm / DSD 1536 mm,
1024 x 768 detector @ 0.4 mm, 720 views over 2 pi.  One step = Siddon forward
projection of all 720 views + matched backprojection of the 720 projections,
device-resident (inputs larger than L2, so no flush is needed).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

value      GRays/s of the Siddon projection (rays of all ranks / max device time)
atb        Gvox-upd/s of the matched backprojection
e2e        the same metrics through the public host API (numpy in, numpy out:
           host->device and device->host copies inside the timed region)
roofline   dominant kernel, algorithmic bytes / CUDA-event duration vs measured HBM
cpu_baseline  the FP64 oracle on a bounded sample of views, all host cores
--impl reference  the reference's own CUDA build (oracle/_ref) through its own
           host-pointer C++ entry points, in a child process
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NV, NU, NA = 768, 1024, 720
NVOX = (512, 512, 512)
DDET, SVOL = 0.4, 256.0
METRIC = "GRays/s Ax + Gvox-upd/s Atb at 512^3"
WORKLOAD = "cone-beam 512^3 @ 0.5 mm, 1024x768 det @ 0.4 mm, 720 views / 2pi, DSO 1000, DSD 1536"
TV_ALPHA, TV_ITERS = 0.002, 20   # POCS-TV timing: 20 descent steps on the phantom volume


def set_size(size, views):
    """--size 256: the 256^3 @ 1 mm / 512x512 @ 0.8 mm case used for profiling captures."""
    global NV, NU, NA, NVOX, DDET, WORKLOAD
    if size == 256:
        NV, NU, NVOX, DDET = 512, 512, (256, 256, 256), 0.8
        WORKLOAD = "cone-beam 256^3 @ 1 mm, 512x512 det @ 0.8 mm, %d views / 2pi, DSO 1000, DSD 1536"
    if views:
        NA = int(views)
    if "%d" in WORKLOAD:
        WORKLOAD = WORKLOAD % NA
    elif views:
        WORKLOAD = WORKLOAD.replace("720 views", "%d views" % NA)


def geometry():
    from tigre_b200.utilities.geometry import cone_geometry
    return cone_geometry(NVOX, (SVOL, SVOL, SVOL), (NV, NU), (DDET, DDET), DSO=1000.0, DSD=1536.0)


def angles():
    return np.linspace(0, 2 * np.pi, NA, endpoint=False).astype(np.float32)


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling (200 ms) during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.fh,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def cpu_baseline(geo, ang, n_views=4):
    """FP64 oracle on n_views evenly spaced views, full detector, all host cores."""
    from oracle import oracle as O
    idx = np.linspace(0, NA, n_views, endpoint=False).astype(int)
    sub = ang[idx]
    img = _phantom_host(0)
    t = time.perf_counter()
    O.ax(img, geo, sub, "Siddon")
    dt = time.perf_counter() - t
    rays = n_views * NU * NV
    return {"value": rays / dt / 1e9, "unit": "GRays/s", "cores": os.cpu_count(), "kind": "port",
            "sample": "FP64 oracle Siddon, %d of %d views, full %dx%d detector, %.1f s" % (n_views, NA, NU, NV, dt)}


def cpu_configs(c2_views=36):
    """The FP64 oracle (all host cores) on the small configurations: C1 (64^3 @ 1 mm, 128x128 @
    0.8 mm, 100 views) in full, and C2 (256^3 @ 1 mm, 512x512 @ 0.8 mm, 360 views over 2 pi) on
    c2_views evenly spaced views, rates extrapolated per ray / per voxel update."""
    from oracle import oracle as O
    from tigre_b200.utilities.geometry import cone_geometry
    from tigre_b200.utilities.phantom import random_ellipsoids
    out = {"impl": "oracle-cpu", "cores": os.cpu_count(), "kind": "port", "configs": {}}
    for name, n, nd, dd, na, nv in (("C1", 64, 128, 0.8, 100, 100), ("C2", 256, 512, 0.8, 360, c2_views)):
        geo = cone_geometry((n, n, n), (float(n),) * 3, (nd, nd), (dd, dd))
        ang = np.linspace(0, 2 * np.pi, na, endpoint=False).astype(np.float32)[
            np.linspace(0, na, nv, endpoint=False).astype(int)]
        img = random_ellipsoids((n, n, n), seed=0)
        rays, upd = nv * nd * nd, nv * n ** 3
        res = {"views_timed": nv, "views": na}
        for op, fn, units, unit in (
                ("ax_siddon", lambda: O.ax(img, geo, ang, "Siddon"), rays, "GRays/s"),
                ("ax_interpolated", lambda: O.ax(img, geo, ang, "interpolated"), rays, "GRays/s")):
            t = time.perf_counter()
            proj = fn()
            dt = time.perf_counter() - t
            res[op] = {"value": round(units / dt / 1e9, 6), "unit": unit, "s": round(dt, 3)}
        for op, kind in (("atb_fdk", "FDK"), ("atb_matched", "matched")):
            t = time.perf_counter()
            O.atb(proj, geo, ang, kind)
            dt = time.perf_counter() - t
            res[op] = {"value": round(upd / dt / 1e9, 6), "unit": "Gvox-upd/s", "s": round(dt, 3)}
        out["configs"][name] = res
    return out


_PH = {}


def _phantom_host(seed):
    if seed not in _PH:
        import torch
        from tigre_b200.utilities.phantom import random_ellipsoids
        dev = "cuda" if torch.cuda.is_available() else "cpu"
        _PH[seed] = random_ellipsoids(NVOX, seed=seed, device=dev).cpu().numpy()
    return _PH[seed]


def conv_layers():
    """Two calls of tigre_conv3d_fwd per U-Net layer shape (128^3 x 16 -> 16 and 64^3 x 64 -> 64,
    random BF16 inputs, ReLU) through the C ABI: the workload of the convolution profile."""
    import ctypes as C
    import torch
    from tigre_b200 import _native as N
    L = N.lib()
    ptr = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
    for n, cin, cout in [(128, 16, 16), (64, 64, 64)]:
        x = torch.randn(n, n, n, cin, device="cuda").to(torch.bfloat16)
        w = (torch.randn(cout, 27 * cin, device="cuda") / 20).to(torch.bfloat16)
        b = torch.zeros(cout, device="cuda")
        y = torch.empty(n, n, n, cout, device="cuda", dtype=torch.bfloat16)
        col = torch.empty(16, dtype=torch.bfloat16, device="cuda")
        for _ in range(2):
            N.check(L.tigre_conv3d_fwd(ptr(x), ptr(w), ptr(b), ptr(y), None, n, n, n, cin, cout, 1, ptr(col), None),
                    "tigre_conv3d_fwd")
        torch.cuda.synchronize()
    print("ok")


def max_over_ranks(dist, values, device):
    """Element-wise maximum of per-rank device times (the slowest rank sets the job time)."""
    import torch
    t = torch.tensor(values, dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()


def job_throughput(world, units_per_rank, seconds):
    """Whole-job rate in G units/s: every replica processes units_per_rank in the max-over-ranks time."""
    return world * units_per_rank / seconds / 1e9


# ------------------------------------------------------------------ CGLS time to residual --
# The learned-vs-plain half of the metric on the warm-start configuration: 256^3 @ 1 mm random
# ellipsoids (seed 0), 512 x 512 detector @ 0.8 mm, 90 views over 2 pi, DSO 1000 / DSD 1536.
C5_VOX, C5_DET, C5_DDET, C5_VIEWS = 256, 512, 0.8, 90
C5_I0 = 5e4
# The metric names 1e-3, but CGLS over TIGRE's operator pair (Siddon Ax, matched Atb: an
# approximate adjoint) stalls above it on this noiseless problem -- its residual starts to grow
# at 3.1e-3 (zero start, 34 iterations; FP64 CGLS over the same pair stalls too), where the
# reference's divergence rule stops it (krylov_subspace_algorithms.py:66-80).  The noiseless
# criterion is therefore 5e-3, the first decade step every start reaches.
C5_TOL = 5e-3
C5_MAX_ITERS = 300
C5_WORKLOAD = ("CGLS on 256^3 @ 1 mm, 512x512 det @ 0.8 mm, 90 views / 2pi, DSO 1000, DSD 1536; "
               "noiseless: Siddon projections of the phantom; noisy: Poisson I0 = 5e4 (+ N(0, 0.5) counts)")


def c5_geometry():
    from tigre_b200.utilities.geometry import cone_geometry
    return cone_geometry((C5_VOX,) * 3, (float(C5_VOX),) * 3, (C5_DET, C5_DET), (C5_DDET, C5_DDET),
                         DSO=1000.0, DSD=1536.0)


def c5_angles():
    return np.linspace(0, 2 * np.pi, C5_VIEWS, endpoint=False).astype(np.float32)


def c5_noise(proj_np):
    """Noisy line integrals with the noise model of CTnoise.add (Python/tigre/utilities/
    CTnoise.py:4-33): counts I0 exp(-p / max p), Poisson plus N(0, 0.5), back to -log(counts /
    I0) max p; drawn with numpy's seeded generator so that both arms of the benchmark get the
    same numbers."""
    p = np.asarray(proj_np, dtype=np.float32)
    pmax = float(p.max())
    rng = np.random.default_rng(1234)
    counts = rng.poisson(C5_I0 * np.exp(-p.astype(np.float64) / pmax)) + rng.normal(0.0, 0.5, p.shape)
    return (-np.log(counts / C5_I0) * pmax).astype(np.float32)


def measure_cgls():
    """Wall time (host clock, synchronised; the whole driver: its per-iteration residual reads
    included) of CGLS until ||b - A x|| / ||b|| meets the criterion, from a zero start and from
    the FDK reconstruction (FDK time included).  Noiseless data: criterion 1e-3.  Noisy data:
    the relative residual stalls at the noise level, so the criterion is the residual of 100
    zero-start iterations + 0.1 %."""
    import torch
    from tigre_b200 import _native as N, projectors as P
    from tigre_b200.algorithms._common import Problem
    from tigre_b200.algorithms.krylov import cgls_device
    from tigre_b200.algorithms.single_pass import fdk_device
    from tigre_b200.utilities.phantom import random_ellipsoids
    from tigre_b200 import warmstart as WS
    geo, ang = c5_geometry(), c5_angles()
    img = random_ellipsoids((C5_VOX,) * 3, seed=0, device="cuda")
    plan = N.get_plan(N.checked_geometry(geo, ang), img.device.index)
    clean = P.ax(img, plan, "Siddon")
    out = {"workload": C5_WORKLOAD}
    model = WS.pretrained_c5()
    if model is not None:
        out["warm_start"] = ("3-D U-Net (4 levels, 16 base channels, BF16, FP32 accumulation) trained by this "
                             "library's kernels on 96 seeded 256^3 phantoms of this configuration (48 noisy at "
                             "I0 = 5e4, 48 noiseless; image loss, then the relative residual after 4-5 unrolled "
                             "CGLS iterations from its output), weights in tigre_b200/data; its inference is "
                             "timed with FDK")
        with torch.no_grad():
            model(torch.zeros((C5_VOX,) * 3, device="cuda"))     # warm-up of the inference kernels

    def run(prob, x0, target):
        torch.cuda.synchronize()
        t = time.perf_counter()
        _, res, _ = cgls_device(prob, C5_MAX_ITERS, x0=x0, tol=target)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t
        rel = np.asarray(res) / prob_bnorm(prob)
        hit = np.nonzero(rel <= target)[0]
        return {"s": round(dt, 4), "iters": int(hit[0]) + 1 if hit.size else len(rel), "reached": bool(hit.size),
                "final_rel_residual": float(rel[-1])}

    def prob_bnorm(prob):
        return float(torch.linalg.vector_norm(prob.b.double()).item())

    for variant in ("noiseless", "noisy"):
        b = clean if variant == "noiseless" else torch.from_numpy(c5_noise(clean.cpu().numpy())).cuda()
        prob = Problem(b, geo, ang)
        cgls_device(prob, 3)                       # warm-up: plan, scratch, pools
        fdk_device(prob)                           # warm-up: the filter's FFT plans
        if variant == "noiseless":
            target, crit = C5_TOL, "||b - Ax|| / ||b|| <= 5e-3 (1e-3 lies below the stall of CGLS over this pair)"
        else:
            _, res100, _ = cgls_device(prob, 100)
            target = float(res100[-1] / prob_bnorm(prob)) * 1.001
            crit = "||b - Ax|| / ||b|| <= 1.001 x its value after 100 zero-start iterations (%.5f)" % target
        row = {"criterion": crit, "target": target, "zero": run(prob, None, target)}
        torch.cuda.synchronize()
        t = time.perf_counter()
        f = fdk_device(prob).clamp_(min=0)
        torch.cuda.synchronize()
        t_fdk = time.perf_counter() - t
        fr = run(prob, f, target)
        fr["fdk_s"] = round(t_fdk, 4)
        fr["s"] = round(fr["s"] + t_fdk, 4)
        row["fdk"] = fr
        if model is not None:
            # learned warm start: FDK, U-Net inference, CGLS from its output (all timed)
            torch.cuda.synchronize()
            t = time.perf_counter()
            with torch.no_grad():
                x0 = (model(fdk_device(prob) * WS.SCALE) / WS.SCALE).contiguous()
            torch.cuda.synchronize()
            t_inf = time.perf_counter() - t
            wr = run(prob, x0, target)
            wr["fdk_and_inference_s"] = round(t_inf, 4)
            wr["s"] = round(wr["s"] + t_inf, 4)
            row["warm"] = wr
            row["warm_over_zero"] = round(wr["s"] / row["zero"]["s"], 3)
            row["warm_over_fdk"] = round(wr["s"] / fr["s"], 3)
        out[variant] = row
    return out


def reference_cgls(T, ref_geo):
    """The reference's own tigre.algorithms.cgls (krylov_subspace_algorithms.py:22-99) on the
    same data, numpy in and out.  It has no tolerance stop: it runs a fixed number of
    iterations, logging ||b - A x|| every iteration with an extra projection; the time to the
    criterion is the run time up to the first iteration that meets it (iterations take equal
    time), or the whole run when none does."""
    from tigre_b200.utilities.phantom import random_ellipsoids
    ang = c5_angles()
    img = np.asarray(random_ellipsoids((C5_VOX,) * 3, seed=0), dtype=np.float32)
    clean = T.Ax(img, ref_geo, ang, "Siddon")
    out = {"workload": C5_WORKLOAD}
    for variant, niter in (("noiseless", 40), ("noisy", 40)):
        b = clean if variant == "noiseless" else c5_noise(clean)
        bnorm = float(np.linalg.norm(b.astype(np.float64)))
        T.algorithms.cgls(b, ref_geo, ang, 2)      # warm-up
        t = time.perf_counter()
        _, l2 = T.algorithms.cgls(b, ref_geo, ang, niter, computel2=True)
        dt = time.perf_counter() - t
        rel = np.asarray(l2, dtype=np.float64).ravel() / bnorm
        out[variant] = {"iters_run": niter, "s_run": round(dt, 3), "s_per_iter": round(dt / niter, 4),
                        "rel_residual": [float(r) for r in rel[:: max(1, niter // 10)]]}
        if variant == "noiseless":
            hit = np.nonzero(rel <= C5_TOL)[0]
            out[variant]["criterion"] = "||b - Ax|| / ||b|| <= %g" % C5_TOL
            out[variant]["reached"] = bool(hit.size)
            if hit.size:
                out[variant]["iters"] = int(hit[0]) + 1
                out[variant]["s"] = round(dt * (int(hit[0]) + 1) / niter, 3)
    return out


def run_reference(args, rank):
    """TIGRE's own package over its own CUDA build for sm_100a (baseline/_ref, made by
    tests/dropin/build.py from the unmodified sources), through its public Python API:
    tigre.Ax / tigre.Atb on numpy arrays, as a TIGRE user calls them."""
    if rank != 0:
        return
    from oracle import reference_package as RP
    if not RP.available("reference"):
        print(json.dumps({"impl": "reference", "unavailable": "stock TIGRE build (baseline/_ref) not present"}))
        return
    T = RP.load("reference")
    geo, ang = RP.geometry_like(T, geometry()), angles()
    img = _phantom_host(0)
    for _ in range(max(1, args.warmup)):
        proj = T.Ax(img, geo, ang, "Siddon")
        T.Atb(proj, geo, ang, "matched")
    t_ax, t_atb = [], []
    for _ in range(args.steps):
        t = time.perf_counter()
        proj = T.Ax(img, geo, ang, "Siddon")
        t_ax.append(time.perf_counter() - t)
        t = time.perf_counter()
        T.Atb(proj, geo, ang, "matched")
        t_atb.append(time.perf_counter() - t)
    rays, upd = NA * NU * NV, NA * math.prod(NVOX)
    v = rays / statistics.median(t_ax) / 1e9
    va = upd / statistics.median(t_atb) / 1e9
    b_in, b_out = math.prod(NVOX) * 4, NA * NU * NV * 4
    line = {
        "impl": "reference", "metric": METRIC, "value": round(v, 4), "unit": "GRays/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(1e3 * (statistics.median(t_ax) + statistics.median(t_atb)), 2),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "reference": "TIGRE's Python package with its Cython extensions and "
                                                      "Common/CUDA built for sm_100a: tigre.Ax(Siddon) + "
                                                      "tigre.Atb(matched) on pageable numpy arrays"},
        "atb": {"value": round(va, 4), "unit": "Gvox-upd/s"},
        "e2e": {"value": round(v, 4), "unit": "GRays/s", "atb_value": round(va, 4), "atb_unit": "Gvox-upd/s",
                "h2d_bytes_per_step": b_in + b_out, "d2h_bytes_per_step": b_out + b_in},
        "cpu_baseline": {"kind": "reference", "cores": os.cpu_count(), "value": round(v, 4), "unit": "GRays/s",
                         "sample": "full workload; the reference has no CPU projector, its CUDA build runs on the GPU"},
    }
    if not args.no_ops:
        ops = {}
        T.Ax(img, geo, ang, "interpolated")
        t = time.perf_counter()
        T.Ax(img, geo, ang, "interpolated")
        dt = time.perf_counter() - t
        ops["ax_interpolated_f32"] = {"value": round(rays / dt / 1e9, 4), "unit": "GRays/s", "ms_per_call": round(1e3 * dt, 3)}
        T.Atb(proj, geo, ang, "FDK")
        t = time.perf_counter()
        T.Atb(proj, geo, ang, "FDK")
        dt = time.perf_counter() - t
        ops["atb_fdk_f32"] = {"value": round(upd / dt / 1e9, 4), "unit": "Gvox-upd/s", "ms_per_call": round(1e3 * dt, 3)}
        from _minTV import minTV
        from tigre.utilities.gpu import GpuIds
        ids = GpuIds()      # the algorithms pass their GpuIds (iterative_recon_alg.py:350)
        minTV(img, TV_ALPHA, TV_ITERS, ids)
        t = time.perf_counter()
        minTV(img, TV_ALPHA, TV_ITERS, ids)
        dt = time.perf_counter() - t
        ops["tv_pocs_f32_e2e"] = {"value": round(math.prod(NVOX) * TV_ITERS / dt / 1e9, 4), "unit": "Gvox-iter/s",
                                  "ms_per_call": round(1e3 * dt, 3)}
        line["ops"] = ops
    if not args.no_cgls:
        line["cgls"] = reference_cgls(T, RP.geometry_like(T, c5_geometry()))
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-ops", action="store_true", help="skip the per-kind kernel timings")
    ap.add_argument("--no-cgls", action="store_true", help="skip the CGLS time-to-residual measurement")
    ap.add_argument("--size", type=int, default=512, choices=[512, 256])
    ap.add_argument("--views", type=int, default=0)
    ap.add_argument("--cpu-configs", action="store_true",
                    help="only time the FP64 CPU oracle on the C1 and C2 configurations and print one JSON line")
    ap.add_argument("--conv-layers", action="store_true",
                    help="only run two forward calls of two U-Net convolution shapes (the conv profile workload)")
    args = ap.parse_args()
    if args.cpu_configs:
        print(json.dumps(cpu_configs()))
        return
    if args.conv_layers:
        conv_layers()
        return
    set_size(args.size, args.views)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    from tigre_b200 import _native as N, projectors as P

    dev = torch.device("cuda", local)
    geo, ang = geometry(), angles()
    plan = N.get_plan(N.checked_geometry(geo, ang), local)
    from tigre_b200.utilities.phantom import random_ellipsoids
    vol = random_ellipsoids(NVOX, seed=rank, device=dev)
    proj = torch.empty((NA, NV, NU), dtype=torch.float32, device=dev)
    bp = torch.empty_like(vol)
    nseg = P.siddon_segments(plan)
    for _ in range(max(3, args.warmup)):
        P.ax(vol, plan, "Siddon", out=proj)
        P.atb(proj, plan, "matched", out=bp)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clk = Clocks(local)
    clk.start()
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(args.steps)]
    torch.cuda.synchronize()
    launches0 = N.lib().tigre_launch_count()
    for k in range(args.steps):
        ev[k][0].record()
        P.ax(vol, plan, "Siddon", out=proj)
        ev[k][1].record()
        P.atb(proj, plan, "matched", out=bp)
        ev[k][2].record()
    torch.cuda.synchronize()
    launches = N.lib().tigre_launch_count() - launches0
    if dist:
        dist.barrier()
    clocks = clk.stop()
    t_ax = sum(e[0].elapsed_time(e[1]) for e in ev) / 1e3
    t_atb = sum(e[1].elapsed_time(e[2]) for e in ev) / 1e3
    t_tot = ev[0][0].elapsed_time(ev[-1][2]) / 1e3
    if dist:
        t_ax, t_atb, t_tot = max_over_ranks(dist, [t_ax, t_atb, t_tot], dev)
    rays = NA * NU * NV
    upd = NA * math.prod(NVOX)
    value = job_throughput(world, rays * args.steps, t_ax)
    atb_value = job_throughput(world, upd * args.steps, t_atb)
    # roofline of the dominant kernel, algorithmic bytes per launch
    peak, peak_kind = peaks()
    ax_launch = t_ax / args.steps
    atb_launch = t_atb / args.steps
    if ax_launch >= atb_launch:
        alg = nseg * 4 + rays * 4           # one voxel gather per Siddon segment + one output write per ray
        rpt = 8 if NV >= 512 else (4 if NV >= 256 else 2)   # rows per thread, as the launcher picks
        roof = {"kernel": "siddon_cells_kernel<float,float,%d>" % rpt, "bound": "hbm",
                "achieved": alg / ax_launch / 1e9, "alg_bytes_per_launch": alg,
                "traffic": _scaled_traffic("siddon", NA), "traffic_source": TRAFFIC_SOURCE,
                "binding": _binding("siddon", ax_launch)}
    else:
        alg = upd * 4 * 4 + math.prod(NVOX) * 4   # 4 bilinear taps per update + one volume write
        roof = {"kernel": "bp_tma_kernel<float,float,true,true>", "bound": "hbm",
                "achieved": alg / atb_launch / 1e9, "alg_bytes_per_launch": alg,
                "traffic": _scaled_traffic("bp", NA), "traffic_source": TRAFFIC_SOURCE,
                "binding": _binding("bp", atb_launch)}
    roof.update({"peak": peak, "unit": "GB/s", "frac": roof["achieved"] / peak, "peak_source": peak_kind})
    for k in ("achieved", "frac"):
        roof[k] = round(roof[k], 4)
    ops = None
    if not args.no_ops:
        ops = time_ops(P, plan, vol, proj)
    e2e = None
    if not args.no_e2e and rank == 0:
        e2e = measure_e2e(vol, geo, ang, min(args.steps, 3))
    cgls = None
    if not args.no_cgls and rank == 0:
        del bp
        cgls = measure_cgls()
    if dist:
        dist.barrier()
    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 4), "unit": "GRays/s", "n_gpus": world, "steps": args.steps,
            "warmup": max(3, args.warmup), "ms_per_step": round(1e3 * t_tot / args.steps, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded random ellipsoids)",
            "config": {"workload": WORKLOAD, "step": "Siddon Ax of %d views + matched Atb of them" % NA,
                       "l2": "inputs larger than L2: no flush (volume %.0f MiB, projections %.2f GiB)" % (
                           math.prod(NVOX) * 4 / 2 ** 20, NA * NU * NV * 4 / 2 ** 30),
                       "parallelism": "replicas" if world > 1 else "single"},
            "atb": {"value": round(atb_value, 4), "unit": "Gvox-upd/s", "ms_per_launch": round(1e3 * atb_launch, 3)},
            "ax_ms_per_launch": round(1e3 * ax_launch, 3),
            "siddon_segments": nseg,
            "roofline": roof,
            "gpu_launches": int(launches),
            "clocks": clocks,
        }
        if ops:
            line["ops"] = ops
        if e2e:
            line["e2e"] = e2e
        if cgls:
            line["cgls"] = cgls
        if not args.no_cpu:
            try:
                line["cpu_baseline"] = cpu_baseline(geo, ang)
            except Exception as ex:  # the baseline must not hide the GPU result
                line["cpu_baseline"] = {"error": str(ex)[:200]}
        print(json.dumps(line))
    if dist:
        dist.destroy_process_group()


# DRAM bytes of one launch on the 512^3 / 1024x768 / 720-view workload, from a single-pass ncu
# capture of that launch (dram__bytes_read.sum + dram__bytes_write.sum;
# profiles/launches_512cube_720views.txt gives the command).  Neither kernel's traffic is
# proportional to the view count (the Siddon grid reuses voxel columns across a tile of 64 views
# in L2; the backprojector reads each view's patches once per voxel block), so the figure is
# reported only for that exact launch.
TRAFFIC_720_VIEWS = {"siddon": 6589300736 + 2287803648, "bp": 22228711168 + 525339136}


TRAFFIC_SOURCE = ("dram__bytes_read.sum + dram__bytes_write.sum of a single-pass ncu capture of the 720-view "
                  "launch on B200 (profiles/launches_512cube_720views.txt), not measured in this run")

# What binds each kernel, from its ncu --set full capture on 36 views of the same workload
# (profiles/siddon_cells_512cube_36views.txt, profiles/bp_tma_matched_512cube_36views.txt): warp
# instructions and shared-memory wavefronts per view of the launch.  The Siddon kernel's DRAM
# traffic is 0.6 % of its algorithmic bytes: it is bound by instruction issue and on-chip load
# latency; the backprojector reads its taps from shared memory: bound by shared wavefronts and issue.
PROFILED = {"siddon": {"warp_inst_per_view": 6.127e9 / 36, "source": "profiles/siddon_cells_512cube_36views.txt"},
            "bp": {"warp_inst_per_view": 2.949e9 / 36, "wavefronts_per_view": 7.605e8 / 36,
                   "ideal_wavefronts_per_view": 512 ** 3 * 4 / 32,
                   "source": "profiles/bp_tma_matched_512cube_36views.txt"}}


def _binding(kind, launch_s):
    """Fraction of the resource that binds the kernel: instruction issue (4 warp instructions per
    SM per clock) for both, and for the backprojector shared-memory wavefronts (1 per SM per
    clock), at the SM clock of the GPU's specification (the clocks key gives the measured one)."""
    if NVOX != (512, 512, 512) or NU != 1024 or NV != 768:
        return None
    sms, hz = 148, 1.965e9
    pr = PROFILED[kind]
    out = {"issue_frac": round(pr["warp_inst_per_view"] * NA / launch_s / (sms * 4 * hz), 4),
           "source": pr["source"] + " (counts per view, scaled to this launch)"}
    if kind == "bp":
        out["resource"] = "shared-memory wavefronts and instruction issue"
        out["shared_wavefront_frac"] = round(pr["wavefronts_per_view"] * NA / launch_s / (sms * hz), 4)
        out["shared_wavefront_floor_ms"] = round(1e3 * pr["ideal_wavefronts_per_view"] * NA / (sms * hz), 2)
    else:
        out["resource"] = "instruction issue and L1/L2 load latency (long-scoreboard stalls)"
    return out


def _scaled_traffic(kind, views):
    exact = NVOX == (512, 512, 512) and NU == 1024 and NV == 768 and views == 720
    return TRAFFIC_720_VIEWS.get(kind) if exact else None


def time_ops(P, plan, vol, proj, reps=3):
    """Kernel-only time per launch of the other projector kinds and of BF16 storage
    (same workload, CUDA events, one untimed launch first)."""
    import torch
    vol16, proj16 = vol.to(torch.bfloat16), proj.to(torch.bfloat16)
    p_out, v_out = torch.empty_like(proj), torch.empty_like(vol)
    p16_out, v16_out = torch.empty_like(proj16), torch.empty_like(vol16)
    rays, upd = NA * NU * NV, NA * math.prod(NVOX)
    cases = {
        "ax_interpolated_f32": (lambda: P.ax(vol, plan, "interpolated", out=p_out), rays, "GRays/s"),
        "atb_fdk_f32": (lambda: P.atb(proj, plan, "FDK", out=v_out), upd, "Gvox-upd/s"),
        "ax_siddon_bf16": (lambda: P.ax(vol16, plan, "Siddon", out=p16_out), rays, "GRays/s"),
        "ax_interpolated_bf16": (lambda: P.ax(vol16, plan, "interpolated", out=p16_out), rays, "GRays/s"),
        "atb_matched_bf16": (lambda: P.atb(proj16, plan, "matched", out=v16_out), upd, "Gvox-upd/s"),
        "atb_fdk_bf16": (lambda: P.atb(proj16, plan, "FDK", out=v16_out), upd, "Gvox-upd/s"),
    }
    tv_vol, tv_work = vol.clone(), torch.empty_like(vol)
    cases["tv_pocs_f32"] = (lambda: P.tv_pocs_(tv_vol, TV_ALPHA, TV_ITERS, tv_work), math.prod(NVOX) * TV_ITERS,
                            "Gvox-iter/s")
    tv_prior = (vol * 0.9).contiguous()
    cases["tv_awtv_f32"] = (lambda: P.tv_aw_pocs_(tv_vol, TV_ALPHA, TV_ITERS, 0.02, tv_work),
                            math.prod(NVOX) * TV_ITERS, "Gvox-iter/s")
    cases["tv_piccs_f32"] = (lambda: P.tv_piccs_(tv_vol, tv_prior, TV_ALPHA, 0.5, TV_ITERS, tv_work),
                             math.prod(NVOX) * TV_ITERS, "Gvox-iter/s")
    from tigre_b200.utilities.im_3d_denoise import tv_denoise_device
    prox_work = torch.empty(5 * NVOX[1] * NVOX[2] * (NVOX[0] + 2), dtype=torch.float32, device=vol.device)
    cases["tv_denoise_f32"] = (lambda: tv_denoise_device(vol, TV_ITERS, 15.0, prox_work), math.prod(NVOX) * TV_ITERS,
                               "Gvox-iter/s")
    # algorithmic bytes per launch (FP32 / BF16 element bytes e): interpolated: 8 corner reads per
    # sample inside the volume + one output write per ray; backprojection: 4 bilinear taps per
    # voxel update + one volume write; POCS-TV: 12 B per voxel and step (norm pass reads f,
    # update pass reads f and writes f'; AwTV the same; PICCS 20 B, the prior read in both passes);
    # TV proximal: 52 B per voxel and iteration (u pass reads f, u, p and writes u; p pass reads
    # u, p and writes p)
    nsamp = P.interp_samples(plan)
    nvox = math.prod(NVOX)
    alg = {"ax_interpolated_f32": nsamp * 8 * 4 + rays * 4, "ax_interpolated_bf16": nsamp * 8 * 2 + rays * 2,
           "atb_fdk_f32": upd * 4 * 4 + nvox * 4, "atb_matched_bf16": upd * 4 * 2 + nvox * 2,
           "atb_fdk_bf16": upd * 4 * 2 + nvox * 2, "tv_pocs_f32": nvox * 12 * TV_ITERS,
           "tv_denoise_f32": nvox * 52 * TV_ITERS, "tv_awtv_f32": nvox * 12 * TV_ITERS,
           "tv_piccs_f32": nvox * 20 * TV_ITERS}
    out = {}
    for name, (fn, units, unit) in cases.items():
        fn()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        dt = e0.elapsed_time(e1) / 1e3 / reps
        out[name] = {"value": round(units / dt / 1e9, 4), "unit": unit, "ms_per_launch": round(1e3 * dt, 3)}
        if name in alg:
            peak = peaks()[0]
            out[name]["alg_gbs"] = round(alg[name] / dt / 1e9, 1)
            out[name]["alg_frac_of_hbm"] = round(alg[name] / dt / 1e9 / peak, 4)
    out["interp_samples"] = nsamp
    del vol16, proj16, p_out, v_out, p16_out, v16_out, tv_vol, tv_work, prox_work, tv_prior
    # POCS-TV through the host API (numpy in and out, copies included), as minTV is called
    from tigre_b200.utilities.minTV import minTV
    host = vol.cpu().numpy()
    minTV(host, TV_ALPHA, TV_ITERS)
    t = time.perf_counter()
    minTV(host, TV_ALPHA, TV_ITERS)
    dt = time.perf_counter() - t
    out["tv_pocs_f32_e2e"] = {"value": round(math.prod(NVOX) * TV_ITERS / dt / 1e9, 4), "unit": "Gvox-iter/s",
                              "ms_per_call": round(1e3 * dt, 3)}
    return out


def measure_e2e(vol, geo, ang, steps):
    """Public host API: numpy in (ordinary pageable arrays, as TIGRE users pass them and as the
    reference arm gets them), numpy out, copies inside the timed region."""
    import tigre_b200 as tigre
    img_np = np.ascontiguousarray(vol.cpu().numpy())
    tigre.Ax(img_np, geo, ang, "Siddon")    # warm-up (plan, pools)
    ta, tb = [], []
    proj_np = None
    for _ in range(steps):
        t = time.perf_counter()
        proj_np = tigre.Ax(img_np, geo, ang, "Siddon")
        ta.append(time.perf_counter() - t)
    proj_in = np.array(proj_np)   # a pageable copy of the projections as the backprojection input
    tigre.Atb(proj_in, geo, ang, "matched")
    for _ in range(steps):
        t = time.perf_counter()
        tigre.Atb(proj_in, geo, ang, "matched")
        tb.append(time.perf_counter() - t)
    # the other two kinds through the same host API (one untimed call first, one timed)
    tigre.Ax(img_np, geo, ang, "interpolated")
    t = time.perf_counter()
    tigre.Ax(img_np, geo, ang, "interpolated")
    ti = time.perf_counter() - t
    tigre.Atb(proj_in, geo, ang, "FDK")
    t = time.perf_counter()
    tigre.Atb(proj_in, geo, ang, "FDK")
    tf = time.perf_counter() - t
    rays, upd = NA * NU * NV, NA * math.prod(NVOX)
    b_vol, b_proj = math.prod(NVOX) * 4, NA * NU * NV * 4
    return {"value": round(rays / statistics.median(ta) / 1e9, 4), "unit": "GRays/s",
            "atb_value": round(upd / statistics.median(tb) / 1e9, 4), "atb_unit": "Gvox-upd/s",
            "ax_s": round(statistics.median(ta), 4), "atb_s": round(statistics.median(tb), 4),
            "interpolated_value": round(rays / ti / 1e9, 4), "fdk_value": round(upd / tf / 1e9, 4),
            "h2d_bytes_per_step": b_vol + b_proj, "d2h_bytes_per_step": b_proj + b_vol}


if __name__ == "__main__":
    main()
