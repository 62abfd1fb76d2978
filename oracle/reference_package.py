"""Importing TIGRE's own Python package as built by tests/dropin/build.py (TEST AND BENCH
INFRASTRUCTURE ONLY): over this library (tests/dropin/_build, for the drop-in tests) or over
the reference's own CUDA build (baseline/_ref, for bench.py's reference arm).

The package imports its plotting modules unconditionally (Python/tigre/__init__.py:51-55 imports
its visualization modules, which import matplotlib at module level).  Neither matplotlib nor
mpl_toolkits is installed here, and nothing on the projector path plots, so a meta-path finder
hands out empty modules whose capitalised attributes are inert classes and whose other
attributes are no-op functions."""
import glob
import importlib.abc
import importlib.machinery
import os
import sys
import types

import numpy as np

_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LOCATIONS = {"ours": os.path.join(_ROOT, "tests", "dropin", "_build"),
             "reference": os.path.join(_ROOT, "baseline", "_ref")}

ROOTS = ("matplotlib", "mpl_toolkits")


class _PlotStub(importlib.abc.MetaPathFinder, importlib.abc.Loader):
    def find_spec(self, name, path, target=None):
        if name.split(".")[0] in ROOTS:
            return importlib.machinery.ModuleSpec(name, self, is_package=True)
        return None

    def create_module(self, spec):
        m = types.ModuleType(spec.name)
        m.__path__ = []

        def attr(a):
            if a.startswith("__"):
                raise AttributeError(a)
            if a[:1].isupper():
                return type(a, (), {"__init__": lambda self, *args, **kw: None})
            return lambda *args, **kw: None

        m.__getattr__ = attr
        return m

    def exec_module(self, module):
        pass


def install():
    if not any(isinstance(f, _PlotStub) for f in sys.meta_path):
        sys.meta_path.insert(0, _PlotStub())


def available(which):
    d = LOCATIONS[which]
    return bool(glob.glob(os.path.join(d, "_Ax*.so"))) and os.path.isdir(os.path.join(d, "tigre"))


def load(which):
    """Imports and returns the `tigre` package of that build (one build per process: both are
    named `tigre` and their extensions `_Ax`, ...)."""
    d = LOCATIONS[which]
    install()
    if d not in sys.path:
        sys.path.insert(0, d)
    import tigre
    if os.path.dirname(tigre.__file__) != os.path.join(d, "tigre"):
        raise ImportError("another tigre package was imported first: %s" % tigre.__file__)
    import tigre.algorithms  # noqa: F401
    return tigre


def geometry_like(T, ours):
    """The package's own geometry object carrying the attributes of one of this library's."""
    g = T.geometry()
    for name in ("mode", "nVoxel", "sVoxel", "dVoxel", "nDetector", "sDetector", "dDetector", "DSO", "DSD",
                 "offOrigin", "offDetector", "rotDetector", "accuracy", "COR"):
        if hasattr(ours, name):
            v = getattr(ours, name)
            setattr(g, name, np.array(v) if isinstance(v, np.ndarray) else v)
    return g
