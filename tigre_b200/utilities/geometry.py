"""Cone-beam geometry model, drop-in for ``tigre.utilities.geometry``.

Same attribute names, array orders and checks as the reference
(Python/tigre/utilities/geometry.py:10-301):

* volume arrays are ``(z, y, x)``: ``nVoxel``, ``sVoxel``, ``dVoxel``;
* detector arrays are ``(v, u)``: ``nDetector``, ``sDetector``, ``dDetector``;
* ``check_geo(angles)`` expands scalars to one value per angle
  (``DSO``, ``DSD``, ``COR`` of shape ``(n,)``; ``offOrigin`` ``(n,3)``;
  ``offDetector`` ``(n,2)``; ``rotDetector`` ``(n,3)``) and turns 1-D angles
  into ``(n, 3)`` ZYZ Euler triples;
* ``cast_to_single()`` casts every float to float32, as the reference does
  before crossing into native code (geometry.py:121-140).
"""
from __future__ import annotations

import numpy as np

__all__ = ["Geometry", "ParallelGeo", "geometry", "ConeGeometryDefault"]

_PER_ANGLE_SCALARS = ("DSD", "DSO", "COR")


class Geometry(object):
    def __init__(self):
        self.mode = None
        self.n_proj = None
        self.angles = None
        self.filter = None
        self.nVoxel = np.zeros(3)
        self.dVoxel = np.zeros(3)
        self.sVoxel = np.zeros(3)
        self.nDetector = np.zeros(2)
        self.dDetector = np.zeros(2)
        self.sDetector = np.zeros(2)

    # -- geometry.py:24-111 -------------------------------------------------
    def check_geo(self, angles, verbose=False):
        angles = np.atleast_1d(np.asarray(angles))
        if angles.ndim == 1:
            self.n_proj = angles.shape[0]
            z = np.zeros((self.n_proj, 1), dtype=np.float32)
            self.angles = np.hstack((angles.reshape(self.n_proj, 1), z, z))
        elif angles.ndim == 2:
            if angles.shape[1] != 3:
                raise BufferError("Expected angles of dimensions (n, 3), got: " + str(angles.shape))
            self.n_proj = angles.shape[0]
            self.angles = angles.copy()
        else:
            raise BufferError("Unexpected angles shape: " + str(angles.shape))
        if self.mode is None:
            self.mode = "cone"

        mandatory = ["nVoxel", "sVoxel", "dVoxel", "nDetector", "sDetector", "dDetector", "DSO", "DSD"]
        missing = [a for a in mandatory if not hasattr(self, a)]
        if missing:
            raise AttributeError("following mandatory fields missing from geometry:" + str(missing))

        for name, shp in (("nVoxel", (3,)), ("sVoxel", (3,)), ("dVoxel", (3,))):
            if not np.shape(getattr(self, name)) == shp:
                raise AttributeError("geo.%s.shape should be (3, )" % name)
        if not sum(abs(self.dVoxel * self.nVoxel - self.sVoxel)) < 1e-6:
            raise AttributeError("nVoxel*dVoxel is not equal to sVoxel. Check fields.")
        for name in ("nDetector", "sDetector", "dDetector"):
            if not np.shape(getattr(self, name)) == (2,):
                raise AttributeError("geo.%s.shape should be (2, )" % name)
        if not sum(abs(self.dDetector * self.nDetector - self.sDetector)) < 1e-6:
            raise AttributeError("nDetector*dDetector is not equal to sDetector. Check fields.")

        for attrib in ("DSD", "DSO"):
            self._repeat_per_angle(attrib, angles)
        defaults = {
            "offOrigin": lambda: np.array([0, 0, 0]),
            "offDetector": lambda: np.array([0, 0]),
            "rotDetector": lambda: np.array([0, 0, 0]),
            "COR": lambda: np.zeros(angles.shape[0]),
        }
        for attrib, make in defaults.items():
            if not hasattr(self, attrib):
                setattr(self, attrib, make())
            self._repeat_per_angle(attrib, angles)
        if not hasattr(self, "accuracy"):
            self.accuracy = 0.5
        if verbose:
            print(str(self))

    def checknans(self):
        for attrib, val in self.__dict__.items():
            if str(val) == "nan":
                raise ValueError("nan found for Geometry attribute:" + attrib)
            if isinstance(val, np.ndarray) and val.dtype.kind == "f" and np.isnan(val).all():
                raise ValueError("Nan found in Geometry attribute:" + attrib)

    # -- geometry.py:121-140 ------------------------------------------------
    def cast_to_single(self):
        exclude = ("nVoxel", "nDetector", "n_proj", "mode", "filter")
        for attrib in list(self.__dict__):
            val = getattr(self, attrib)
            if val is None or attrib in exclude:
                continue
            try:
                arr = np.array(val)
                if np.issubdtype(arr.dtype, np.integer):
                    continue
                setattr(self, attrib, np.float32(val))
            except (ValueError, TypeError):
                pass

    # -- geometry.py:142-211 ------------------------------------------------
    def _repeat_per_angle(self, attrib, angles):
        old = getattr(self, attrib)
        n = angles.shape[0]
        if type(old) in (float, int, np.float32, np.float64, np.int32, np.int64):
            setattr(self, attrib, np.tile(old, n))
        elif isinstance(old, np.ndarray):
            if old.ndim == 1:
                if old.shape in ((3,), (2,)) and attrib not in _PER_ANGLE_SCALARS:
                    setattr(self, attrib, np.tile(old, (n, 1)))
                elif old.shape == (1,):
                    if attrib in _PER_ANGLE_SCALARS:
                        setattr(self, attrib, np.tile(old, n))
                    else:
                        setattr(self, attrib, np.tile(old, (n, 1)))
                elif old.shape == (n,):
                    pass
            elif old.ndim == 0:
                setattr(self, attrib, np.tile(old, n))
            else:
                if old.shape != (n, old.shape[1]):
                    raise AttributeError(
                        "%s with shape: %s not compatible with shapes: %s"
                        % (attrib, old.shape, [(n,), (n, old.shape[1]), (3,), (2,), (1,)]))
        else:
            raise TypeError("Data type not understood for: geo.%s with type = %s" % (attrib, type(old)))

    # kept for scripts written against the reference's private name
    __check_and_repmat__ = _repeat_per_angle

    def __str__(self):
        lines = ["TIGRE parameters", "-----", "Geometry parameters",
                 "Distance from source to detector (DSD) = %s mm" % (self.DSD,),
                 "Distance from source to origin (DSO)= %s mm" % (self.DSO,),
                 "-----", "Detector parameters",
                 "Number of pixels (nDetector) = %s" % (self.nDetector,),
                 "Size of each pixel (dDetector) = %s mm" % (self.dDetector,),
                 "Total size of the detector (sDetector) = %s mm" % (self.sDetector,),
                 "-----", "Image parameters",
                 "Number of voxels (nVoxel) = %s" % (self.nVoxel,),
                 "Total size of the image (sVoxel) = %s mm" % (self.sVoxel,),
                 "Size of each voxel (dVoxel) = %s mm" % (self.dVoxel,)]
        if hasattr(self, "accuracy"):
            lines.append("Samples per pixel of forward projection (accuracy) = %s" % (self.accuracy,))
        return "\n".join(lines)


class ParallelGeo(Geometry):
    """Parallel-beam geometry (geometry.py:274-301).  The parallel projectors
    are not part of this build; the native entry points return an error."""

    def __init__(self, nVoxel):  # noqa: N803
        if nVoxel is None:
            raise ValueError("nVoxel needs to be given for initialisation of parallel beam")
        Geometry.__init__(self)
        self.mode = "parallel"
        self.nVoxel = nVoxel
        self.dVoxel = np.array([1, 1, 1])
        self.sVoxel = self.nVoxel
        self.DSO = np.float32(self.nVoxel[0])
        self.DSD = np.float32(self.nVoxel[0] * 2)
        self.dDetector = np.array([1, 1])
        self.nDetector = np.zeros((2,), dtype=np.int64)
        self.nDetector[0] = self.nVoxel[0]
        self.nDetector[1] = max(self.nVoxel[1], self.nVoxel[2])
        self.sDetector = self.nDetector
        self.accuracy = 0.5
        self.offOrigin = np.array([0, 0, 0])
        self.offDetector = np.array([0, 0])
        self.rotDetector = np.array([0, 0, 0])


class ConeGeometryDefault(Geometry):
    """Default cone-beam geometry (geometry_default.py:7-80)."""

    def __init__(self, high_resolution=True, nVoxel=None):  # noqa: N803
        Geometry.__init__(self)
        self.DSD = 1536.0
        self.DSO = 1000.0
        if high_resolution:
            self.nDetector = np.array((512, 512))
            self.dDetector = np.array((0.8, 0.8))
            self.nVoxel = np.array((512, 512, 512))
        else:
            self.nDetector = np.array((128, 128))
            self.dDetector = np.array((0.8, 0.8)) * 4
            self.nVoxel = np.array((64, 64, 64))
        if nVoxel is not None:
            self.nDetector = np.array((nVoxel[1], nVoxel[2]))
            self.dDetector = np.array([0.8, 0.8])
            self.nVoxel = np.array(nVoxel)
        self.sDetector = self.nDetector * self.dDetector
        self.sVoxel = np.array((256, 256, 256))
        self.dVoxel = self.sVoxel / self.nVoxel
        self.offOrigin = np.array((0, 0, 0))
        self.offDetector = np.array((0, 0))
        self.rotDetector = np.array((0, 0, 0))
        self.accuracy = 0.5
        self.mode = "cone"
        self.filter = None


def geometry(mode="cone", nVoxel=None, default=False, high_resolution=True):  # noqa: N803
    """Constructor with the reference's signature (geometry.py:303-348)."""
    if mode == "cone":
        if default:
            return ConeGeometryDefault(high_resolution, nVoxel)
        return Geometry()
    if mode == "parallel":
        return ParallelGeo(nVoxel)
    raise ValueError("mode: " + mode + " not recognized.")


def cone_geometry(nVoxel, sVoxel, nDetector, dDetector, DSO=1000.0, DSD=1536.0, accuracy=0.5):  # noqa: N803
    """Convenience builder used by the tests and benchmarks (not in the reference API)."""
    g = Geometry()
    g.mode = "cone"
    g.DSO = float(DSO)
    g.DSD = float(DSD)
    g.nVoxel = np.array(nVoxel, dtype=np.int64)
    g.sVoxel = np.array(sVoxel, dtype=np.float64)
    g.dVoxel = g.sVoxel / g.nVoxel
    g.nDetector = np.array(nDetector, dtype=np.int64)
    g.dDetector = np.array(dDetector, dtype=np.float64)
    g.sDetector = g.nDetector * g.dDetector
    g.offOrigin = np.array((0.0, 0.0, 0.0))
    g.offDetector = np.array((0.0, 0.0))
    g.rotDetector = np.array((0.0, 0.0, 0.0))
    g.accuracy = accuracy
    return g
