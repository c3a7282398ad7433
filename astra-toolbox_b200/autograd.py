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
device, float32 / float16 / bfloat16, with optional leading batch
dimensions.  A float32 batch of small problems (up to BATCH_MAX_VOXELS voxels
each) is projected in one persistent launch per direction (b2t_batch3d_fp
and its exact adjoint b2t_batch3d_matched_bp: the items of a batch are one
packed buffer as they are); larger or 16-bit items go through the
single-problem projectors one by one, each of which fills the GPU.
"""
import numpy as np
import torch

from . import _lib
from .batch import Batch3D
from .projector import Projector3D

# Largest item (voxels) projected through the batched kernels.
BATCH_MAX_VOXELS = 128 ** 3


def _fp(projector, vol):
    out = torch.empty(projector.proj_shape, device=vol.device, dtype=vol.dtype)
    projector.fp(vol.contiguous(), out)
    return out


def _at(projector, proj):
    out = torch.empty(projector.vol_shape, device=proj.device, dtype=proj.dtype)
    projector.bp(proj.contiguous(), out, kernel=_lib.KER_MATCHED_BP)
    return out


def _batch_plan(projector, n):
    """The Batch3D of n copies of this projector's problem, or None when the
    items go one by one (see the module docstring)."""
    if projector.is_cyl or projector.vox_ss != 1:
        return None
    nvox, nproj = int(np.prod(projector.vol_shape)), int(np.prod(projector.proj_shape))
    if nvox > BATCH_MAX_VOXELS or nvox % 32 or nproj % 32:
        return None  # (packed items start on 32-element boundaries)
    cache = projector.__dict__.setdefault('_batch3d', {})
    if n not in cache:
        opts = {'DetectorSuperSampling': projector.det_ss}
        cache[n] = Batch3D([(projector.proj_geom, projector.vol_geom, opts)] * n)
    return cache[n]


def _batched(fn, projector, x, base_ndim):
    if x.dim() == base_ndim:
        return fn(projector, x)
    out_shape = projector.proj_shape if fn is _fp else projector.vol_shape
    items = x.reshape(-1, *x.shape[-base_ndim:])
    B = _batch_plan(projector, items.shape[0]) if x.dtype == torch.float32 else None
    if B is not None:
        flat = items.contiguous().view(-1)
        with torch.cuda.device(x.device):
            out = B.fp(flat) if fn is _fp else B.bp(flat, matched=True)
        return out.view(*x.shape[:-base_ndim], *out_shape)
    return torch.stack([fn(projector, xi) for xi in items]).reshape(*x.shape[:-base_ndim], *out_shape)


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
