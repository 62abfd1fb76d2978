"""Build TIGRE's own Python package on top of libtigre_b200.so (test infrastructure only).

    python tests/dropin/build.py [--force]          # CPU only; needs the TIGRE source tree

This is the drop-in that the C ABI promises, done the way a maintainer of TIGRE would do it:
the reference's Python package (Python/tigre, copied unmodified into tests/dropin/_build/,
which git ignores) gets its eight Cython extensions (top-level modules _Ax, _Atb, ..., beside
the package, as the reference's setup.py installs them) compiled from the reference's own
unmodified .pyx files, with the extension blocks of the reference's setup.py:347-509 except
that the CUDA sources of the projectors and regularisers (Siddon_projection.cu,
voxel_backprojection*.cu, GD_TV.cu, ...) are replaced by linking libtigre_b200.so, which
exports the same C++ symbols (include/tigre_b200_compat.hpp).  The host-side helpers that the
extensions compile in the reference build are kept from the TIGRE tree (GpuIds.cpp,
gpuUtils.cu).  Nothing here runs at test time: tests/test_dropin_gpu.py imports the result.

The TIGRE tree is read in place from $TIGRE_REFERENCE (default /root/reference); without it this
script does nothing.
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
OUT = os.path.join(HERE, "_build")
PKG = os.path.join(OUT, "tigre")
PYX_DIR = os.path.join(PKG, "utilities", "cuda_interface")
OBJ = os.path.join(OUT, "obj")
REFERENCE_ROOT = os.environ.get("TIGRE_REFERENCE", "/root/reference")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA, "bin", "nvcc")
LIB_DIR = os.path.join(ROOT, "tigre_b200")

# extension -> (pyx, host helpers of the TIGRE tree it compiles in the reference build,
#               whether it links libtigre_b200.so); setup.py:347-509
EXTENSIONS = {
    "_Ax": ("_Ax.pyx", ["GpuIds.cpp"], True),
    "_Atb": ("_Atb.pyx", ["GpuIds.cpp", "gpuUtils.cu"], True),
    "_tv_proximal": ("_tv_proximal.pyx", ["GpuIds.cpp", "gpuUtils.cu"], True),
    "_minTV": ("_minTV.pyx", ["GpuIds.cpp", "gpuUtils.cu"], True),
    "_minPICCS": ("_minPICCS.pyx", ["GpuIds.cpp", "gpuUtils.cu"], True),
    "_AwminTV": ("_AwminTV.pyx", ["GpuIds.cpp", "gpuUtils.cu"], True),
    "_gpuUtils": ("_gpuUtils.pyx", ["gpuUtils.cu"], False),
    "_RandomNumberGenerator": ("_randomNumberGenerator.pyx", ["GpuIds.cpp", "gpuUtils.cu"], True),
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


def build(force: bool = False) -> list[str]:
    """Returns the built extension paths ([] when the TIGRE tree is absent)."""
    if not available():
        return []
    import numpy as np
    cuda_src = os.path.join(REFERENCE_ROOT, "Common", "CUDA")
    if force and os.path.isdir(PKG):
        shutil.rmtree(PKG)
    if not os.path.isdir(PKG):
        shutil.copytree(os.path.join(REFERENCE_ROOT, "Python", "tigre"), PKG,
                        ignore=shutil.ignore_patterns("*.so", "__pycache__", "*.c", "*.cpp"))
    os.makedirs(OBJ, exist_ok=True)
    suffix = sysconfig.get_config_var("EXT_SUFFIX")
    inc = ["-I" + sysconfig.get_paths()["include"], "-I" + np.get_include(), "-I" + os.path.join(CUDA, "include"),
           "-I" + cuda_src]
    defs = ["-DIS_FOR_PYTIGRE", "-DNPY_NO_DEPRECATED_API=NPY_1_7_API_VERSION"]
    # host helpers, once
    helpers = {}
    for f in ("GpuIds.cpp", "gpuUtils.cu"):
        src = os.path.join(cuda_src, f)
        obj = os.path.join(OBJ, f.replace(".", "_") + ".o")
        if force or _stale(obj, [src]):
            if f.endswith(".cu"):
                _run([NVCC, "-O2", "-Xcompiler", "-fPIC", *defs, *inc, "-c", src, "-o", obj])
            else:
                _run(["g++", "-O2", "-fPIC", "-std=c++17", *defs, *inc, "-c", src, "-o", obj])
        helpers[f] = obj
    lib = os.path.join(LIB_DIR, "libtigre_b200.so")
    # the extensions are top-level modules (setup.py names them "_Ax", ...; tigre/utilities/Ax.py
    # imports "from _Ax import _Ax_ext"), so they sit in tests/dropin/_build, three levels below
    # the repository
    rpath = "$ORIGIN/../../../tigre_b200"

    def one(name):
        pyx_name, extra, link_ours = EXTENSIONS[name]
        pyx = os.path.join(PYX_DIR, pyx_name)
        cpp = os.path.join(OBJ, name + ".cpp")
        so = os.path.join(OUT, name + suffix)
        deps = [pyx] + [helpers[e] for e in extra] + ([lib] if link_ours else [])
        if not (force or _stale(so, deps)):
            return so
        _run([sys.executable, "-m", "cython", "--cplus", "-3", "--module-name", name, "-I", OUT, pyx, "-o", cpp])
        cmd = ["g++", "-O2", "-fPIC", "-shared", "-std=c++17", "-w", *defs, *inc, cpp,
               *[helpers[e] for e in extra], "-o", so, "-L" + os.path.join(CUDA, "lib64"), "-lcudart",
               "-Wl,-rpath," + os.path.join(CUDA, "lib64")]
        if link_ours:
            cmd += ["-L" + LIB_DIR, "-ltigre_b200", "-Wl,-rpath," + rpath]
        _run(cmd)
        return so

    with ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        return list(ex.map(one, EXTENSIONS))


if __name__ == "__main__":
    for p in build(force="--force" in sys.argv):
        print(p)
