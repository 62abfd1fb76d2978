"""Build recipe for the checker libraries (test infrastructure only).

* ``oracle/_build/liboracle.so`` -- the FP64 host oracle (oracle.cpp), g++ + OpenMP.
* ``oracle/_ref/libref_{ax,atb,tv}.so`` -- the reference's own CUDA projectors,
  compiled for sm_100a straight from the TIGRE source tree (read in place,
  never copied into this repository) plus the extern "C" shim ref_shim.cpp.
  The three groups follow the reference's extension blocks (setup.py:347-433),
  because the reference defines helpers such as checkFreeMemory in several
  translation units and they only link cleanly in those groups.

Run ``python oracle/build.py`` (or ``__graft_entry__.build()``).
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
REF_OUT = os.path.join(HERE, "_ref")
# the TIGRE source tree (read in place); TIGRE_REFERENCE overrides where it lives
REFERENCE_ROOT = os.environ.get("TIGRE_REFERENCE", "/root/reference")
REFERENCE_CUDA = os.path.join(REFERENCE_ROOT, "Common", "CUDA")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

# the reference's own extension groupings (setup.py:347-433)
REF_GROUPS = {
    "ax": (["projection.cpp", "TIGRE_common.cpp", "GpuIds.cpp", "Siddon_projection.cu",
            "Siddon_projection_parallel.cu", "ray_interpolated_projection.cu",
            "ray_interpolated_projection_parallel.cu"], "REF_AX"),
    "atb": (["TIGRE_common.cpp", "GpuIds.cpp", "gpuUtils.cu", "voxel_backprojection.cu",
             "voxel_backprojection2.cu", "voxel_backprojection_parallel.cu"], "REF_ATB"),
    "tv": (["TIGRE_common.cpp", "GpuIds.cpp", "gpuUtils.cu", "GD_TV.cu"], "REF_TV"),
    # a separate extension in the reference too (_tv_proximal): it repeats helpers of GD_TV.cu
    "prox": (["TIGRE_common.cpp", "GpuIds.cpp", "gpuUtils.cu", "tv_proximal.cu"], "REF_PROX"),
    # _AwminTV and _minPICCS are separate extensions too (each repeats GD_TV.cu's helpers)
    "awtv": (["TIGRE_common.cpp", "GpuIds.cpp", "gpuUtils.cu", "GD_AwTV.cu"], "REF_AWTV"),
    "piccs": (["TIGRE_common.cpp", "GpuIds.cpp", "gpuUtils.cu", "PICCS.cu"], "REF_PICCS"),
}


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("command failed: %s\n%s\n%s" % (" ".join(cmd), r.stdout, r.stderr))
    return r


def _newer(out, srcs):
    if not os.path.exists(out):
        return False
    t = os.path.getmtime(out)
    return all(os.path.getmtime(s) <= t for s in srcs)


def build_oracle(force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    src = os.path.join(HERE, "oracle.cpp")
    out = os.path.join(BUILD, "liboracle.so")
    if force or not _newer(out, [src]):
        _run(["g++", "-O2", "-std=c++17", "-fopenmp", "-shared", "-fPIC", src, "-o", out])
    return out


def build_ref(force: bool = False) -> list[str]:
    """Compile the reference CUDA groups; returns the built paths ([] if the TIGRE tree is absent)."""
    if not os.path.isdir(REFERENCE_CUDA):
        return []
    os.makedirs(REF_OUT, exist_ok=True)
    objdir = os.path.join(REF_OUT, "obj")
    os.makedirs(objdir, exist_ok=True)
    shim = os.path.join(HERE, "ref_shim.cpp")
    common = ["-DIS_FOR_PYTIGRE", "-I" + REFERENCE_CUDA]
    jobs = {}
    for name, (files, _) in REF_GROUPS.items():
        for f in files:
            src = os.path.join(REFERENCE_CUDA, f)
            obj = os.path.join(objdir, f.replace(".", "_") + ".o")
            if f.endswith(".cu"):
                # flags of setup.py:32-36 (per-thread default stream) for sm_100a
                cmd = [NVCC, *ARCH, "-O3", "--default-stream=per-thread", "-Xcompiler", "-fPIC",
                       *common, "-c", src, "-o", obj]
            else:
                cmd = ["g++", "-O2", "-fPIC", *common, "-I/usr/local/cuda/include", "-c", src, "-o", obj]
            jobs[obj] = (cmd, [src])
    outs = []
    with ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        futs = [ex.submit(_run, c) for o, (c, s) in jobs.items() if force or not _newer(o, s)]
        for f in futs:
            f.result()
    for name, (files, macro) in REF_GROUPS.items():
        shim_obj = os.path.join(objdir, "shim_%s.o" % name)
        if force or not _newer(shim_obj, [shim]):
            _run(["g++", "-O2", "-fPIC", "-D" + macro, *common, "-I/usr/local/cuda/include", "-c", shim,
                  "-o", shim_obj])
        objs = [os.path.join(objdir, f.replace(".", "_") + ".o") for f in files] + [shim_obj]
        out = os.path.join(REF_OUT, "libref_%s.so" % name)
        if force or not _newer(out, objs):
            _run([NVCC, *ARCH, "-shared", "-o", out, *objs])
        outs.append(out)
    return outs


if __name__ == "__main__":
    print(build_oracle(force="--force" in sys.argv))
    print(build_ref(force="--force" in sys.argv))
