"""Run the reference's own CUDA projectors (oracle/_ref, built by oracle/build.py).

TEST INFRASTRUCTURE ONLY: used by tests/ (golden fixtures, reference parity)
and by bench.py's reference arm.  The reference exits the process on any CUDA
error (Common/CUDA/TIGRE_common.cpp:13-16) and pocs_tv resets the device
(GD_TV.cu:681), so every call runs in a fresh child process; inputs and
outputs travel through .npy files in a temporary directory.

    from oracle import ref
    out, seconds = ref.ax(img, geo, angles, "Siddon")        # numpy in/out
"""
from __future__ import annotations

import copy
import ctypes as C
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

_FP = C.POINTER(C.c_float)


class Geometry(C.Structure):
    # layout of struct Geometry, Common/CUDA/types_TIGRE.hpp:48-85
    _fields_ = [
        ("nVoxelX", C.c_int), ("nVoxelY", C.c_int), ("nVoxelZ", C.c_int),
        ("sVoxelX", C.c_float), ("sVoxelY", C.c_float), ("sVoxelZ", C.c_float),
        ("dVoxelX", C.c_float), ("dVoxelY", C.c_float), ("dVoxelZ", C.c_float),
        ("offOrigX", _FP), ("offOrigY", _FP), ("offOrigZ", _FP), ("DSO", _FP),
        ("nDetecU", C.c_int), ("nDetecV", C.c_int),
        ("sDetecU", C.c_float), ("sDetecV", C.c_float), ("dDetecU", C.c_float), ("dDetecV", C.c_float),
        ("offDetecU", _FP), ("offDetecV", _FP), ("DSD", _FP), ("dRoll", _FP), ("dPitch", _FP), ("dYaw", _FP),
        ("unitX", C.c_float), ("unitY", C.c_float), ("unitZ", C.c_float),
        ("alpha", C.c_float), ("theta", C.c_float), ("psi", C.c_float),
        ("COR", _FP), ("maxLength", C.c_float), ("accuracy", C.c_float),
    ]


def available() -> bool:
    return all(os.path.exists(os.path.join(REF_DIR, "libref_%s.so" % g)) for g in ("ax", "atb", "tv", "prox", "awtv", "piccs"))


def _geo_dict(geo, angles):
    g = copy.deepcopy(geo)
    g.check_geo(angles)
    g.cast_to_single()
    n = g.angles.shape[0]
    f = lambda v, shp: np.asarray(v, dtype=np.float32).reshape(shp).tolist()  # noqa: E731
    return {
        "nVoxel": [int(v) for v in g.nVoxel], "sVoxel": f(g.sVoxel, 3), "dVoxel": f(g.dVoxel, 3),
        "nDetector": [int(v) for v in g.nDetector], "sDetector": f(g.sDetector, 2), "dDetector": f(g.dDetector, 2),
        "DSO": f(g.DSO, n), "DSD": f(g.DSD, n), "offOrigin": f(g.offOrigin, (n, 3)),
        "offDetector": f(g.offDetector, (n, 2)), "rotDetector": f(g.rotDetector, (n, 3)), "COR": f(g.COR, n),
        "accuracy": float(g.accuracy), "angles": f(g.angles, (n, 3)),
    }


def _c_geometry(d, keep):
    n = len(d["DSO"])

    def arr(v):
        a = np.ascontiguousarray(np.asarray(v, dtype=np.float32).reshape(n))
        keep.append(a)
        return a.ctypes.data_as(_FP)

    off, offd, rot = np.array(d["offOrigin"]), np.array(d["offDetector"]), np.array(d["rotDetector"])
    s = Geometry()
    s.nVoxelX, s.nVoxelY, s.nVoxelZ = d["nVoxel"][2], d["nVoxel"][1], d["nVoxel"][0]
    s.sVoxelX, s.sVoxelY, s.sVoxelZ = d["sVoxel"][2], d["sVoxel"][1], d["sVoxel"][0]
    s.dVoxelX, s.dVoxelY, s.dVoxelZ = d["dVoxel"][2], d["dVoxel"][1], d["dVoxel"][0]
    s.offOrigX, s.offOrigY, s.offOrigZ = arr(off[:, 2]), arr(off[:, 1]), arr(off[:, 0])
    s.DSO = arr(d["DSO"])
    s.nDetecU, s.nDetecV = d["nDetector"][1], d["nDetector"][0]
    s.sDetecU, s.sDetecV = d["sDetector"][1], d["sDetector"][0]
    s.dDetecU, s.dDetecV = d["dDetector"][1], d["dDetector"][0]
    s.offDetecU, s.offDetecV = arr(offd[:, 1]), arr(offd[:, 0])
    s.DSD = arr(d["DSD"])
    s.dRoll, s.dPitch, s.dYaw = arr(rot[:, 2]), arr(rot[:, 1]), arr(rot[:, 0])
    s.unitX = s.unitY = s.unitZ = 1.0
    s.COR = arr(d["COR"])
    s.accuracy = d["accuracy"]
    return s


def _worker(spec_path):
    """Child process: load one reference library, run `repeat` calls, save output + timings."""
    spec = json.load(open(spec_path))
    keep = []
    geo = _c_geometry(spec["geo"], keep) if "geo" in spec else None
    inp = np.ascontiguousarray(np.load(spec["input"]), dtype=np.float32)
    dev = int(spec.get("device", 0))
    times = []
    op = spec["op"]
    if op in ("siddon", "interpolated"):
        L = C.CDLL(os.path.join(REF_DIR, "libref_ax.so"))
        L.ref_ax.argtypes = [C.c_void_p, C.POINTER(Geometry), C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int]
        ang = np.ascontiguousarray(np.array(spec["geo"]["angles"], dtype=np.float32))
        n = ang.shape[0]
        out = np.empty((n, geo.nDetecV, geo.nDetecU), dtype=np.float32)
        for _ in range(int(spec.get("repeat", 1))):
            t = time.perf_counter()
            kind = (0 if op == "siddon" else 1) + (2 if spec.get("parallel") else 0)
            rc = L.ref_ax(inp.ctypes.data, C.byref(geo), out.ctypes.data, ang.ctypes.data, n, kind, dev)
            times.append(time.perf_counter() - t)
            if rc:
                raise SystemExit("reference returned %d" % rc)
    elif op in ("fdk", "matched"):
        L = C.CDLL(os.path.join(REF_DIR, "libref_atb.so"))
        L.ref_atb.argtypes = [C.c_void_p, C.POINTER(Geometry), C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int]
        ang = np.ascontiguousarray(np.array(spec["geo"]["angles"], dtype=np.float32))
        n = ang.shape[0]
        out = np.empty((geo.nVoxelZ, geo.nVoxelY, geo.nVoxelX), dtype=np.float32)
        for _ in range(int(spec.get("repeat", 1))):
            t = time.perf_counter()
            kind = 2 if spec.get("parallel") else (0 if op == "fdk" else 1)
            rc = L.ref_atb(inp.ctypes.data, C.byref(geo), out.ctypes.data, ang.ctypes.data, n, kind, dev)
            times.append(time.perf_counter() - t)
            if rc:
                raise SystemExit("reference returned %d" % rc)
    elif op == "pocs_tv":
        L = C.CDLL(os.path.join(REF_DIR, "libref_tv.so"))
        L.ref_pocs_tv.argtypes = [C.c_void_p, C.c_void_p, C.c_float, C.c_void_p, C.c_int, C.c_int]
        out = np.empty_like(inp)
        size = (C.c_long * 3)(inp.shape[2], inp.shape[1], inp.shape[0])
        for _ in range(int(spec.get("repeat", 1))):
            t = time.perf_counter()
            L.ref_pocs_tv(inp.ctypes.data, out.ctypes.data, float(spec["alpha"]), C.cast(size, C.c_void_p),
                          int(spec["maxiter"]), dev)
            times.append(time.perf_counter() - t)
    elif op == "tvdenoise":
        L = C.CDLL(os.path.join(REF_DIR, "libref_prox.so"))
        L.ref_tvdenoise.argtypes = [C.c_void_p, C.c_void_p, C.c_float, C.c_void_p, C.c_int, C.c_int]
        out = np.empty_like(inp)
        size = (C.c_long * 3)(inp.shape[2], inp.shape[1], inp.shape[0])
        for _ in range(int(spec.get("repeat", 1))):
            t = time.perf_counter()
            L.ref_tvdenoise(inp.ctypes.data, out.ctypes.data, float(spec["lmbda"]), C.cast(size, C.c_void_p),
                            int(spec["maxiter"]), dev)
            times.append(time.perf_counter() - t)
    elif op == "aw_pocs_tv":
        L = C.CDLL(os.path.join(REF_DIR, "libref_awtv.so"))
        L.ref_aw_pocs_tv.argtypes = [C.c_void_p, C.c_void_p, C.c_float, C.c_void_p, C.c_int, C.c_float, C.c_int]
        out = np.empty_like(inp)
        size = (C.c_long * 3)(inp.shape[2], inp.shape[1], inp.shape[0])
        for _ in range(int(spec.get("repeat", 1))):
            t = time.perf_counter()
            L.ref_aw_pocs_tv(inp.ctypes.data, out.ctypes.data, float(spec["alpha"]), C.cast(size, C.c_void_p),
                             int(spec["maxiter"]), float(spec["delta"]), dev)
            times.append(time.perf_counter() - t)
    elif op == "piccs_tv":
        L = C.CDLL(os.path.join(REF_DIR, "libref_piccs.so"))
        L.ref_piccs_tv.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_float, C.c_float, C.c_void_p, C.c_int,
                                   C.c_int]
        prior = np.ascontiguousarray(np.load(spec["prior"]), dtype=np.float32)
        out = np.empty_like(inp)
        size = (C.c_long * 3)(inp.shape[2], inp.shape[1], inp.shape[0])
        for _ in range(int(spec.get("repeat", 1))):
            t = time.perf_counter()
            L.ref_piccs_tv(inp.ctypes.data, prior.ctypes.data, out.ctypes.data, float(spec["alpha"]),
                           float(spec["ratio"]), C.cast(size, C.c_void_p), int(spec["maxiter"]), dev)
            times.append(time.perf_counter() - t)
    else:
        raise SystemExit("unknown op " + op)
    np.save(spec["output"], out)
    json.dump({"seconds": times}, open(spec["timing"], "w"))


def _run(op, inp, geo=None, angles=None, repeat=1, device=0, timeout=1800, **extra):
    if not available():
        raise RuntimeError("reference build missing in oracle/_ref (run oracle/build.py where the TIGRE tree exists)")
    with tempfile.TemporaryDirectory() as td:
        spec = {"op": op, "input": os.path.join(td, "in.npy"), "output": os.path.join(td, "out.npy"),
                "timing": os.path.join(td, "t.json"), "repeat": repeat, "device": device}
        spec.update(extra)
        if geo is not None:
            spec["geo"] = _geo_dict(geo, angles)
        np.save(spec["input"], np.ascontiguousarray(inp, dtype=np.float32))
        if "prior_array" in extra:
            spec.pop("prior_array")
            spec["prior"] = os.path.join(td, "prior.npy")
            np.save(spec["prior"], np.ascontiguousarray(extra["prior_array"], dtype=np.float32))
        sp = os.path.join(td, "spec.json")
        json.dump(spec, open(sp, "w"))
        r = subprocess.run([sys.executable, os.path.abspath(__file__), "--worker", sp], capture_output=True,
                           text=True, timeout=timeout)
        if r.returncode != 0:
            raise RuntimeError("reference %s failed (rc=%d):\n%s\n%s" % (op, r.returncode, r.stdout[-2000:],
                                                                          r.stderr[-2000:]))
        return np.load(spec["output"]), json.load(open(spec["timing"]))["seconds"]


def ax(img, geo, angles, projection_type="Siddon", repeat=1, device=0):
    op = "interpolated" if projection_type == "interpolated" else "siddon"
    return _run(op, img, geo, angles, repeat=repeat, device=device,
                parallel=getattr(geo, "mode", "cone") == "parallel")


def atb(proj, geo, angles, backprojection_type="FDK", repeat=1, device=0):
    op = "matched" if backprojection_type == "matched" else "fdk"
    return _run(op, proj, geo, angles, repeat=repeat, device=device,
                parallel=getattr(geo, "mode", "cone") == "parallel")


def pocs_tv(img, alpha, maxiter, repeat=1, device=0):
    return _run("pocs_tv", img, alpha=float(alpha), maxiter=int(maxiter), repeat=repeat, device=device)



def tvdenoise(img, lmbda, maxiter, repeat=1, device=0):
    """The reference's tvdenoising on img (already scaled as im3ddenoise scales it)."""
    return _run("tvdenoise", img, lmbda=float(lmbda), maxiter=int(maxiter), repeat=repeat, device=device)


def aw_pocs_tv(img, alpha, maxiter, delta, repeat=1, device=0):
    """The reference's aw_pocs_tv (AwminTV)."""
    return _run("aw_pocs_tv", img, alpha=float(alpha), maxiter=int(maxiter), delta=float(delta), repeat=repeat,
                device=device)


def piccs_tv(img, prior, alpha, ratio, maxiter, repeat=1, device=0):
    """The reference's piccs_tv (minPICCS)."""
    return _run("piccs_tv", img, alpha=float(alpha), ratio=float(ratio), maxiter=int(maxiter), repeat=repeat,
                device=device, prior_array=prior)


if __name__ == "__main__":
    if len(sys.argv) == 3 and sys.argv[1] == "--worker":
        _worker(sys.argv[2])
    else:
        print(__doc__)
