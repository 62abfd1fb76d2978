"""torch.autograd Functions over the device projector pair and TV.

Replaces the reference's bindings (Python/tigre/utilities/pytorch_bindings.py:9-158),
which round-trip every call through host numpy and use the FDK backprojector as
the backward of Ax (:64).  Here everything stays on the GPU and:

* AxFunction.backward = matched backprojection (A^T), the adjoint pair;
* AtbFunction.backward = Siddon forward projection, the adjoint of the matched
  backprojector.  The FDK backprojector's weights (DSO/U)^2 have no forward
  counterpart here, so AtbFunction accepts only backprojection_type "matched";
  FDK backprojection is a reconstruction step, not an operator to differentiate;
* TVFunction.forward = sum_i |grad f_i| (the TV of pocs_tv's boundary rule),
  backward = grad_output * dTV/df from the hand-written gradient kernel
  (GD_TV.cu:117-143 formula).

Leading batch dimensions are supported by looping over them (one kernel
launch per volume).
"""
from __future__ import annotations

import itertools

import torch

from . import _native as N
from . import projectors as P


def _batched(fn, x, out_shape, dtype=torch.float32):
    lead = x.shape[:-3]
    out = torch.empty(tuple(lead) + tuple(out_shape), dtype=dtype, device=x.device)
    for idx in itertools.product(*[range(d) for d in lead]):
        out[idx] = fn(x[idx].contiguous())
    return out


class AxFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, vol, plan, projection_type="Siddon"):
        ctx.plan = plan
        shape = (plan.n,) + plan.det_shape
        return _batched(lambda v: P.ax(v, plan, projection_type, out_dtype=torch.float32), vol.detach(), shape)

    @staticmethod
    def backward(ctx, g):
        plan = ctx.plan
        gv = _batched(lambda p: P.atb(p.float(), plan, "matched", out_dtype=torch.float32), g.contiguous(),
                      plan.vol_shape)
        return gv, None, None


class AtbFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, proj, plan, backprojection_type="matched"):
        if backprojection_type != "matched":
            raise ValueError("AtbFunction differentiates the matched backprojector only (its adjoint is the "
                             "Siddon projector); got backprojection_type=%r" % (backprojection_type,))
        ctx.plan = plan
        return _batched(lambda p: P.atb(p, plan, backprojection_type, out_dtype=torch.float32), proj.detach(),
                        plan.vol_shape)

    @staticmethod
    def backward(ctx, g):
        plan = ctx.plan
        shape = (plan.n,) + plan.det_shape
        gp = _batched(lambda v: P.ax(v.float(), plan, "Siddon", out_dtype=torch.float32), g.contiguous(), shape)
        return gp, None, None


class TVFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, vol):
        vol = vol.detach().float().contiguous()
        ctx.save_for_backward(vol)
        lead = vol.shape[:-3]
        vals = [P.tv_value(vol[idx]) for idx in itertools.product(*[range(d) for d in lead])]
        return torch.stack(vals).sum().to(torch.float32)

    @staticmethod
    def backward(ctx, g):
        (vol,) = ctx.saved_tensors
        grad = _batched(lambda v: P.tv_gradient(v), vol, vol.shape[-3:])
        return grad * g


class A(torch.nn.Module):
    """Forward operator module (reference: pytorch_bindings.A)."""

    def __init__(self, geo, angles, gpuids=None, projection_type="Siddon"):
        super().__init__()
        dev = 0 if not gpuids else int(list(getattr(gpuids, "devices", gpuids))[0])
        self.plan = N.get_plan(N.checked_geometry(geo, angles), dev)
        self.projection_type = projection_type

    def forward(self, x):
        return AxFunction.apply(x, self.plan, self.projection_type)


class At(torch.nn.Module):
    """Adjoint (matched backprojection) module (reference: pytorch_bindings.At)."""

    def __init__(self, geo, angles, gpuids=None, backprojection_type="matched"):
        super().__init__()
        if backprojection_type != "matched":
            raise ValueError("At is the matched backprojector (the adjoint of the Siddon A); "
                             "got backprojection_type=%r" % (backprojection_type,))
        dev = 0 if not gpuids else int(list(getattr(gpuids, "devices", gpuids))[0])
        self.plan = N.get_plan(N.checked_geometry(geo, angles), dev)
        self.backprojection_type = backprojection_type

    def forward(self, y):
        return AtbFunction.apply(y, self.plan, self.backprojection_type)


def tv(vol):
    return TVFunction.apply(vol)


def create_pytorch_operator(geo, angles, gpuids=None):
    """(A, At) modules, as pytorch_bindings.create_pytorch_operator."""
    return A(geo, angles, gpuids), At(geo, angles, gpuids)
