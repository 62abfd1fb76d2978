"""tigre_b200 -- B200-native (sm_100a) TIGRE projector pair and the iterations built on it.

Drop-in names of the reference package (Python/tigre/__init__.py):

    import tigre_b200 as tigre
    geo = tigre.geometry(mode="cone", default=True, nVoxel=np.array([256, 256, 256]))
    proj = tigre.Ax(img, geo, angles, "Siddon")          # or "interpolated"
    vol = tigre.Atb(proj, geo, angles, "matched")        # or "FDK"
    rec = tigre.algorithms.cgls(proj, geo, angles, niter=10)

numpy arguments take the reference's host path (host pointers through the
C ABI); CUDA torch tensors stay on the device.
"""
from .utilities.geometry import geometry, Geometry, ParallelGeo, cone_geometry  # noqa: F401
from .utilities.geometry import ConeGeometryDefault as geometry_default  # noqa: F401
from .utilities.Ax import Ax  # noqa: F401
from .utilities.Atb import Atb  # noqa: F401
from .utilities.minTV import minTV  # noqa: F401
from .utilities.AwminTV import AwminTV  # noqa: F401
from .utilities.minPICCS import minPICCS  # noqa: F401
from .utilities.gpu import GpuIds, getGpuIds, getGpuNames  # noqa: F401

__version__ = "1.0.0"


def __getattr__(name):
    # heavier submodules are imported on first use
    if name in ("algorithms", "projectors", "autograd"):
        import importlib
        mod = importlib.import_module("." + name, __name__)
        globals()[name] = mod
        return mod
    raise AttributeError(name)
