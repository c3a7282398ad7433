"""Multi-GPU angle partitioning of the 3D projection operators, one process per
GPU (torch.distributed; NCCL over NVLink on GPUs, gloo on CPU).

The reference splits work across GPUs inside CompositeGeometryManager: FP jobs
by projection blocks and BP jobs by volume blocks, with no exchange between
GPUs (src/CompositeGeometryManager.cpp:262-268,1358-1379), and its iterative
algorithms run on one GPU.  Here the views are partitioned:

- every rank holds the whole volume and a contiguous block of the views
  (`view_range`), i.e. its own rows of A;
- FP is local: a rank projects only its views (no communication);
- BP sums every rank's partial backprojection with one all-reduce of the
  volume;
- SIRT keeps the replicated volume consistent because every rank applies the
  same all-reduced update; the line weights are local, the pixel weights are
  one all-reduced BP of ones (src/CudaSirtAlgorithm3D.cpp:261-296), and the
  residual norm sums the ranks' squared norms.

Per-rank compute is any object with `fp(vol, proj)` / `bp(proj, vol)` (SET
semantics), `vol_shape` and `proj_shape` for the rank's sub-geometry; by
default the GPU Projector3D.
"""
import copy

import numpy as np
import torch
import torch.distributed as dist

from ._lib import AstraError


def view_range(n_views, world, rank):
    """Contiguous, balanced block of views of `rank`: [start, stop)."""
    if world <= 0 or not (0 <= rank < world):
        raise AstraError(1, "bad rank %d of %d" % (rank, world))
    base, extra = divmod(n_views, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def shard_proj_geom(proj_geom, start, stop):
    """The projection geometry of views [start, stop) of a 3D proj_geom."""
    t = proj_geom['type']
    g = copy.deepcopy(proj_geom)
    if t in ('cone', 'parallel3d'):
        g['ProjectionAngles'] = np.asarray(proj_geom['ProjectionAngles'])[start:stop].copy()
    elif t in ('cone_vec', 'parallel3d_vec', 'cyl_cone_vec'):
        g['Vectors'] = np.asarray(proj_geom['Vectors'])[start:stop].copy()
    else:
        raise AstraError(2, "angle sharding needs a 3D projection geometry, got %r" % t)
    return g


def _world(group):
    if dist.is_available() and dist.is_initialized():
        return dist.get_world_size(group), dist.get_rank(group)
    return 1, 0


def _gpu_projector(proj_geom, vol_geom):
    from .projector import Projector3D
    return Projector3D(proj_geom, vol_geom)


class AngleShardedOperator:
    """This rank's rows of the 3D projection operator A (its block of views).

    fp(vol, proj_local): proj_local = A_rank vol (local, no communication).
    bp(proj_local, vol): vol = sum over ranks of each rank's BP (all-reduce).
    """

    def __init__(self, proj_geom, vol_geom, group=None, projector_factory=None):
        self.group = group
        self.world, self.rank = _world(group)
        key = 'ProjectionAngles' if 'ProjectionAngles' in proj_geom else 'Vectors'
        self.start, self.stop = view_range(len(proj_geom[key]), self.world, self.rank)
        self.local_geom = shard_proj_geom(proj_geom, self.start, self.stop)
        self.op = (projector_factory or _gpu_projector)(self.local_geom, vol_geom)
        self.vol_shape = self.op.vol_shape
        self.proj_shape = self.op.proj_shape  # local: (det rows, local views, det cols)

    def allreduce(self, t):
        if self.world > 1:
            dist.all_reduce(t, op=dist.ReduceOp.SUM, group=self.group)
        return t

    def fp(self, vol, proj_local):
        self.op.fp(vol, proj_local)
        return proj_local

    def bp(self, proj_local, vol):
        self.op.bp(proj_local, vol)
        return self.allreduce(vol)


def _invert(t):
    """opInvert (cuda/3d/arith3d.cu:87-94): 1/x where x > 1e-6, else 0."""
    return torch.where(t > 1e-6, 1.0 / t.clamp_min(1e-30), torch.zeros_like(t))


class ShardedSIRT:
    """SIRT3D_CUDA over angle-sharded ranks (CudaSirtAlgorithm3D.cpp:261-381):
    x += lambda W_pix (sum_r B_r W_line,r (b_r - A_r x)), with optional min /
    max constraints.  `sino_local` is this rank's block of views."""

    def __init__(self, op, relaxation=1.0, min_constraint=None, max_constraint=None):
        self.op = op
        self.relaxation = float(relaxation)
        self.min_c = min_constraint
        self.max_c = max_constraint
        self.line_w = None
        self.pix_w = None

    def _weights(self, like_vol, like_proj):
        line = torch.empty_like(like_proj)
        self.op.fp(torch.ones_like(like_vol), line)
        self.line_w = _invert(line)
        pix = torch.empty_like(like_vol)
        self.op.bp(torch.ones_like(like_proj), pix)
        self.pix_w = _invert(pix) * self.relaxation

    def run(self, sino_local, vol, iterations):
        if self.line_w is None:
            self._weights(vol, sino_local)
        r = torch.empty_like(sino_local)
        d = torch.empty_like(vol)
        for _ in range(int(iterations)):
            self.op.fp(vol, r)
            r.sub_(sino_local).neg_().mul_(self.line_w)
            self.op.bp(r, d)
            vol.addcmul_(self.pix_w, d)
            if self.min_c is not None:
                vol.clamp_(min=float(self.min_c))
            if self.max_c is not None:
                vol.clamp_(max=float(self.max_c))
        return vol

    def residual_norm(self, sino_local, vol):
        """||b - A x||_2 over all ranks' views (FP64 accumulation)."""
        r = torch.empty_like(sino_local)
        self.op.fp(vol, r)
        sq = torch.tensor([float(((sino_local.double() - r.double()) ** 2).sum())], dtype=torch.float64,
                          device=vol.device)
        self.op.allreduce(sq)
        return float(sq.sqrt().item())
