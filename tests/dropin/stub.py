"""Import-time stand-ins for the plotting packages that TIGRE's Python package imports
unconditionally (Python/tigre/__init__.py:51-55 imports its visualization modules, which import
matplotlib at module level).  Neither matplotlib nor mpl_toolkits is installed here, and nothing
on the projector path plots, so a meta-path finder hands out empty modules whose capitalised
attributes are inert classes and whose other attributes are no-op functions."""
import importlib.abc
import importlib.machinery
import sys
import types

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
