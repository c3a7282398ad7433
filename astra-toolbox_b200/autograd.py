"""Differentiable projectors: torch.autograd Functions over libb2tomo.

ForwardProjection.apply(vol, projector) = A vol, with the exact adjoint A^T
(projection kernel matched_bp: the transpose of the ray-driven forward
projector, sample for sample) as its backward.  BackProjection is the exact
adjoint as a forward op, with A as its backward.  The pair passes the
dot-product test <A x, y> = <x, A^T y> to rounding.

The reference has no autograd; its BP (voxel-driven, ray-density weighted) is
not the adjoint of its FP (the reference's own tests accept a 10 % mismatch,
tests/python/functional/test_rec_scaling.py:147-174).  `astra_bp_gradient`
returns the gradient one would get by using that BP in place of A^T, so its
deviation from the exact gradient can be measured.

Volumes are (z, y, x) and projections (v, angle, u) tensors on a CUDA
device, float32 / float16 / bfloat16; a leading batch dimension is projected
item by item.
"""
import torch

from . import _lib
from .projector import Projector3D


def _fp(projector, vol):
    out = torch.empty(projector.proj_shape, device=vol.device, dtype=vol.dtype)
    projector.fp(vol.contiguous(), out)
    return out


def _at(projector, proj):
    out = torch.empty(projector.vol_shape, device=proj.device, dtype=proj.dtype)
    projector.bp(proj.contiguous(), out, kernel=_lib.KER_MATCHED_BP)
    return out


def _batched(fn, projector, x, base_ndim):
    if x.dim() == base_ndim:
        return fn(projector, x)
    return torch.stack([fn(projector, xi) for xi in x.reshape(-1, *x.shape[-base_ndim:])]).reshape(
        *x.shape[:-base_ndim], *(projector.proj_shape if fn is _fp else projector.vol_shape))


class ForwardProjection(torch.autograd.Function):
    """y = A x; dL/dx = A^T dL/dy (exact adjoint)."""

    @staticmethod
    def forward(ctx, vol, projector):
        if not isinstance(projector, Projector3D):
            raise TypeError("projector must be a Projector3D")
        ctx.projector = projector
        return _batched(_fp, projector, vol, 3)

    @staticmethod
    def backward(ctx, grad):
        return _batched(_at, ctx.projector, grad, 3), None


class BackProjection(torch.autograd.Function):
    """x = A^T y; dL/dy = A dL/dx."""

    @staticmethod
    def forward(ctx, proj, projector):
        ctx.projector = projector
        return _batched(_at, projector, proj, 3)

    @staticmethod
    def backward(ctx, grad):
        return _batched(_fp, ctx.projector, grad, 3), None


def forward_project(vol, projector):
    return ForwardProjection.apply(vol, projector)


def back_project(proj, projector):
    return BackProjection.apply(proj, projector)


def astra_bp_gradient(projector, grad_proj):
    """The reference-style 'gradient' B g using ASTRA's unmatched BP (default kernel)."""
    out = torch.empty(projector.vol_shape, device=grad_proj.device, dtype=grad_proj.dtype)
    projector.bp(grad_proj.contiguous(), out, kernel=_lib.KER_DEFAULT)
    return out
