"""GPU selection, drop-in for tigre.utilities.gpu (Python/tigre/utilities/gpu.py:12-58)."""
from __future__ import annotations

import copy


def _device_names():
    try:
        import torch
        if torch.cuda.is_available():
            return [torch.cuda.get_device_name(i) for i in range(torch.cuda.device_count())]
    except Exception:
        pass
    return []


class GpuIds(object):
    """IDs of the GPUs whose name matches nameGPU (all GPUs when empty/None)."""

    def __init__(self, nameGPU=None):  # noqa: N803
        self.name = "" if nameGPU is None else nameGPU
        names = _device_names()
        self.devices = [i for i, n in enumerate(names) if not self.name or n == self.name]

    def __len__(self):
        return len(self.devices)

    def __str__(self):
        return {"name": self.name, "devices": self.devices}.__str__()

    def __getitem__(self, key):
        one = copy.deepcopy(self)
        one.devices = [self.devices[key]]
        return one


def getGpuNames():  # noqa: N802
    return _device_names()


def getGpuIds(gpuName=None):  # noqa: N802,N803
    return GpuIds(gpuName)


def device_list(gpuids):
    """Plain list of device ids from a GpuIds object, a list, or None (device 0)."""
    if gpuids is None:
        return [0]
    devs = getattr(gpuids, "devices", gpuids)
    devs = [int(d) for d in devs]
    return devs or [0]
