"""Build TIGRE's own Python package with its Cython extensions (test and bench infrastructure).

    python tests/dropin/build.py [--force]          # CPU only; needs the TIGRE source tree

Two builds of the same unmodified package (Python/tigre, copied, never committed) and of its
eight Cython extensions (top-level modules _Ax, _Atb, ..., beside the package, as the
reference's setup.py installs them), compiled from the reference's own .pyx files with the
extension blocks of its setup.py:347-509:

* backend "ours" -> tests/dropin/_build/: the drop-in that the C ABI promises.  The CUDA
  sources of the projectors and regularisers (Siddon_projection.cu, voxel_backprojection*.cu,
  GD_TV.cu, ...) are replaced by linking libtigre_b200.so, which exports the same C++
  symbols (include/tigre_b200_compat.hpp).  tests/test_dropin_gpu.py imports it.
* backend "reference" -> baseline/_ref/: the stock reference, every extension compiled with
  its own CUDA sources for sm_100a (the flags of setup.py:32-36), as `pip install` would
  build it on this GPU.  bench.py's reference arm imports it.

Both keep the host-side helpers the extensions compile in the reference build (GpuIds.cpp,
gpuUtils.cu, TIGRE_common.cpp, projection.cpp) from the TIGRE tree, which is read in place
from $TIGRE_REFERENCE (default /root/reference); without it this script does nothing.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
import sysconfig
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = {"ours": os.path.join(HERE, "_build"), "reference": os.path.join(ROOT, "baseline", "_ref")}
REFERENCE_ROOT = os.environ.get("TIGRE_REFERENCE", "/root/reference")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
LIB_DIR = os.path.join(ROOT, "tigre_b200")

# extension -> (pyx, sources of the reference's Extension block, setup.py:347-509).  The
# backend "ours" keeps the host helpers and links libtigre_b200.so instead of the rest.
HOST_HELPERS = ("GpuIds.cpp", "gpuUtils.cu", "TIGRE_common.cpp", "projection.cpp")
EXTENSIONS = {
    "_Ax": ("_Ax.pyx", ["projection.cpp", "TIGRE_common.cpp", "Siddon_projection.cu",
                        "Siddon_projection_parallel.cu", "ray_interpolated_projection.cu",
                        "ray_interpolated_projection_parallel.cu", "GpuIds.cpp"]),
    "_Atb": ("_Atb.pyx", ["TIGRE_common.cpp", "voxel_backprojection.cu", "voxel_backprojection2.cu",
                          "voxel_backprojection_parallel.cu", "GpuIds.cpp", "gpuUtils.cu"]),
    "_tv_proximal": ("_tv_proximal.pyx", ["TIGRE_common.cpp", "tv_proximal.cu", "GpuIds.cpp", "gpuUtils.cu"]),
    "_minTV": ("_minTV.pyx", ["TIGRE_common.cpp", "GD_TV.cu", "GpuIds.cpp", "gpuUtils.cu"]),
    "_minPICCS": ("_minPICCS.pyx", ["TIGRE_common.cpp", "PICCS.cu", "GpuIds.cpp", "gpuUtils.cu"]),
    "_AwminTV": ("_AwminTV.pyx", ["TIGRE_common.cpp", "GD_AwTV.cu", "GpuIds.cpp", "gpuUtils.cu"]),
    "_gpuUtils": ("_gpuUtils.pyx", ["gpuUtils.cu"]),
    "_RandomNumberGenerator": ("_randomNumberGenerator.pyx", ["TIGRE_common.cpp", "RandomNumberGenerator.cu",
                                                             "GpuIds.cpp", "gpuUtils.cu"]),
}


def _run(cmd, cwd=None):
    r = subprocess.run(cmd, capture_output=True, text=True, cwd=cwd)
    if r.returncode != 0:
        raise RuntimeError("command failed: %s\n%s\n%s" % (" ".join(cmd), r.stdout, r.stderr))
    return r


def _stale(out, deps):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def available():
    return os.path.isdir(os.path.join(REFERENCE_ROOT, "Python", "tigre"))


def _sources(backend, srcs):
    if backend == "ours":
        return [s for s in srcs if s in HOST_HELPERS and s not in ("TIGRE_common.cpp", "projection.cpp")]
    return list(srcs)


def build(backend: str = "ours", force: bool = False) -> list[str]:
    """Returns the built extension paths ([] when the TIGRE tree is absent)."""
    if not available():
        return []
    import numpy as np
    out = OUT[backend]
    pkg = os.path.join(out, "tigre")
    pyx_dir = os.path.join(pkg, "utilities", "cuda_interface")
    obj_dir = os.path.join(out, "obj")
    cuda_src = os.path.join(REFERENCE_ROOT, "Common", "CUDA")
    if force and os.path.isdir(pkg):
        shutil.rmtree(pkg)
    if not os.path.isdir(pkg):
        shutil.copytree(os.path.join(REFERENCE_ROOT, "Python", "tigre"), pkg,
                        ignore=shutil.ignore_patterns("*.so", "__pycache__", "*.c", "*.cpp"))
    os.makedirs(obj_dir, exist_ok=True)
    suffix = sysconfig.get_config_var("EXT_SUFFIX")
    inc = ["-I" + sysconfig.get_paths()["include"], "-I" + np.get_include(), "-I" + os.path.join(CUDA, "include"),
           "-I" + cuda_src]
    defs = ["-DIS_FOR_PYTIGRE", "-DNPY_NO_DEPRECATED_API=NPY_1_7_API_VERSION"]
    # objects of the TIGRE sources, once each
    needed = sorted({f for _, srcs in EXTENSIONS.values() for f in _sources(backend, srcs)})
    objs = {}

    def compile_one(f):
        src = os.path.join(cuda_src, f)
        obj = os.path.join(obj_dir, f.replace(".", "_") + ".o")
        if force or _stale(obj, [src]):
            if f.endswith(".cu"):
                # setup.py:32-36: per-thread default stream; device code for this GPU only
                _run([NVCC, *ARCH, "-O3", "--default-stream=per-thread", "-Xcompiler", "-fPIC", *defs, *inc,
                      "-c", src, "-o", obj])
            else:
                _run(["g++", "-O2", "-fPIC", "-std=c++17", *defs, *inc, "-c", src, "-o", obj])
        return f, obj

    with ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        objs.update(dict(ex.map(compile_one, needed)))
    lib = os.path.join(LIB_DIR, "libtigre_b200.so")
    # the extensions sit three levels below the repository (tests/dropin/_build, baseline/_ref)
    rpath = "$ORIGIN/../../../tigre_b200" if backend == "ours" else None

    def one(name):
        pyx_name, srcs = EXTENSIONS[name]
        mine = [objs[f] for f in _sources(backend, srcs)]
        link_ours = backend == "ours" and name != "_gpuUtils"
        pyx = os.path.join(pyx_dir, pyx_name)
        cpp = os.path.join(obj_dir, name + ".cpp")
        so = os.path.join(out, name + suffix)
        deps = [pyx] + mine + ([lib] if link_ours else [])
        if not (force or _stale(so, deps)):
            return so
        _run([sys.executable, "-m", "cython", "--cplus", "-3", "--module-name", name, "-I", out, pyx, "-o", cpp])
        cmd = ["g++", "-O2", "-fPIC", "-shared", "-std=c++17", "-w", *defs, *inc, cpp, *mine, "-o", so,
               "-L" + os.path.join(CUDA, "lib64"), "-lcudart", "-Wl,-rpath," + os.path.join(CUDA, "lib64")]
        if link_ours:
            cmd += ["-L" + LIB_DIR, "-ltigre_b200", "-Wl,-rpath," + rpath]
        _run(cmd)
        return so

    with ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        return list(ex.map(one, EXTENSIONS))


if __name__ == "__main__":
    for b in ("ours", "reference"):
        for p in build(b, force="--force" in sys.argv):
            print(p)
