"""Shared plumbing of the device-resident algorithm drivers."""
from __future__ import annotations

import copy

import numpy as np

from .. import _native as N
from ..utilities.gpu import device_list


def torch():
    import torch as _t
    return _t


class Problem:
    """Projections, geometry and plan of one reconstruction, resident on one GPU.

    numpy inputs are copied to the device once; results go back as numpy.
    CUDA tensors stay where they are and results are tensors.
    """

    def __init__(self, proj, geo, angles, gpuids=None):
        T = torch()
        self.numpy_in = not (type(proj).__module__.startswith("torch"))
        if self.numpy_in:
            dev = device_list(gpuids)[0]
            self.device = T.device("cuda", dev)
            self.b = T.from_numpy(np.ascontiguousarray(proj, dtype=np.float32)).to(self.device)
        else:
            self.device = proj.device
            self.b = proj.detach().to(T.float32).contiguous()
        self.geo_in = geo
        # checked at the caller's precision: geometries derived from this one (view subsets, the
        # ART weight geometries) are re-checked by Ax/Atb, and a float32 copy of
        # sDetector = nDetector * dDetector can miss check_geo's 1e-6 size test
        self.geo_full = copy.deepcopy(geo)
        self.geo_full.check_geo(angles)
        self.geo = N.checked_geometry(geo, angles)
        self.angles = np.ascontiguousarray(np.asarray(self.geo.angles, dtype=np.float32).reshape(-1, 3))
        self.n = self.angles.shape[0]
        want = (self.n, int(self.geo.nDetector[0]), int(self.geo.nDetector[1]))
        if tuple(self.b.shape) != want:
            raise ValueError("Expected data shape: %s not compatible with: %s" % (want, tuple(self.b.shape)))
        self.plan = N.get_plan(self.geo, self.device.index)
        self.vol_shape = tuple(int(v) for v in self.geo.nVoxel)

    def zeros_vol(self):
        T = torch()
        return T.zeros(self.vol_shape, dtype=T.float32, device=self.device)

    def to_device_vol(self, x):
        T = torch()
        if type(x).__module__.startswith("torch"):
            return x.detach().to(self.device, T.float32).contiguous().clone()
        x = np.ascontiguousarray(x, dtype=np.float32)
        if x.shape != self.vol_shape:
            raise ValueError("wrong dimension of array for initialization")
        return T.from_numpy(x).to(self.device)

    def out(self, x):
        return x.cpu().numpy() if self.numpy_in else x

    def sub_geometry(self, index):
        """Geometry restricted to the views in `index` (art_data_minimizing, iterative_recon_alg.py:326-345)."""
        g = copy.deepcopy(self.geo_full)
        idx = np.asarray(index)
        for name in ("offOrigin", "offDetector", "rotDetector", "DSD", "DSO", "COR"):
            setattr(g, name, np.asarray(getattr(self.geo_full, name))[idx])
        g.angles = self.angles[idx]
        return g

    def contiguous_range(self, index):
        idx = np.asarray(index).reshape(-1)
        if idx.size and np.all(np.diff(idx) == 1):
            return int(idx[0]), int(idx[-1]) + 1
        return None
