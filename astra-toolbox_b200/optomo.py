"""astra.OpTomo: a projector as a linear operator (python/astra/optomo.py).

`W = OpTomo(proj_id)`; `W * x` forward-projects, `W.T * s` backprojects, and W
works in scipy.sparse.linalg solvers (lsqr, cgls-style methods) as the
reference's does.  Differences, both additive: the work runs directly on the
projector's libb2tomo calls instead of creating FP/BP algorithm objects per
product, and CUDA torch tensors are accepted and returned as CUDA tensors
(no host round trip), so the operator also serves torch-side solvers.
"""
import numpy as np
import scipy.sparse.linalg
import torch

from . import algorithm as _alg
from . import data2d as _d2
from . import data3d as _d3
from . import projector as _P


class OpTomo(scipy.sparse.linalg.LinearOperator):
    """The projection matrix of a 'cuda' or 'cuda3d' projector."""

    def __init__(self, proj_id):
        self.pr = _P.lookup_projector(proj_id)
        self.proj_id = proj_id
        self.is3d = isinstance(self.pr, _P.Projector3D)
        self.vg = self.pr.vol_geom
        self.pg = self.pr.proj_geom
        self.vshape = tuple(self.pr.vol_shape)
        self.sshape = tuple(self.pr.proj_shape)
        self.vsize = int(np.prod(self.vshape))
        self.ssize = int(np.prod(self.sshape))
        self.data_mod = _d3 if self.is3d else _d2
        self.appendString = ("3D" if self.is3d else "") + "_CUDA"
        super().__init__(np.float32, (self.ssize, self.vsize))
        self.transposeOpTomo = OpTomoTranspose(self)

    def _transpose(self):
        return self.transposeOpTomo

    _adjoint = _transpose

    # -- products ------------------------------------------------------------
    def _device(self):
        return self.pr.device()

    def _apply(self, x, in_shape, out_shape, forward, out=None):
        is_torch = isinstance(x, torch.Tensor)
        dev = self._device()
        if is_torch and x.is_cuda:
            t = x.reshape(in_shape).to(torch.float32).contiguous()
        else:
            arr = x.detach().cpu().numpy() if is_torch else np.asarray(x)
            t = torch.from_numpy(np.ascontiguousarray(arr.reshape(in_shape), dtype=np.float32)).to(dev)
        res = torch.empty(out_shape, dtype=torch.float32, device=t.device)
        if forward:
            self.pr.fp(t, res)
        else:
            self.pr.bp(t, res)
        if is_torch and x.is_cuda:
            return res
        res = res.cpu().numpy()
        if out is not None:
            out[...] = res.reshape(out.shape)
            return out
        return res

    def FP(self, v, out=None):
        """Forward projection of v (any shape holding the volume's elements)."""
        return self._apply(v, self.vshape, self.sshape, True, out)

    def BP(self, s, out=None):
        """Backprojection of s (any shape holding the projection data's elements)."""
        return self._apply(s, self.sshape, self.vshape, False, out)

    def _matvec(self, v):
        r = self.FP(v)
        return r.reshape(-1)

    def rmatvec(self, s):
        r = self.BP(s)
        return r.reshape(-1)

    def _rmatvec(self, s):
        return self.rmatvec(s)

    def __mul__(self, v):
        # a 2D / 3D volume (or a CUDA tensor) projects directly
        if isinstance(v, torch.Tensor) or (isinstance(v, np.ndarray) and v.shape == self.vshape):
            return self.FP(v)
        return scipy.sparse.linalg.LinearOperator.__mul__(self, v)

    def reconstruct(self, method, s, iterations=1, extraOptions=None):
        """Run a _CUDA reconstruction algorithm on s with this projector and
        return the reconstruction (OpTomo.reconstruct)."""
        if not method.endswith('_CUDA'):
            method = method + ('3D_CUDA' if self.is3d and not method.endswith('3D') else '_CUDA')
        arr = s.detach().cpu().numpy() if isinstance(s, torch.Tensor) else np.asarray(s)
        sid = self.data_mod.create('-proj3d' if self.is3d else '-sino', self.pg,
                                   np.ascontiguousarray(arr.reshape(self.sshape), dtype=np.float32))
        vid = self.data_mod.create('-vol', self.vg, 0)
        cfg = _alg.astra_dict(method)
        cfg['ProjectionDataId'] = sid
        cfg['ReconstructionDataId'] = vid
        cfg['ProjectorId'] = self.proj_id
        cfg['option'] = dict(extraOptions or {})
        aid = _alg.create(cfg)
        try:
            _alg.run(aid, iterations)
            return self.data_mod.get(vid)
        finally:
            _alg.delete(aid)
            self.data_mod.delete([vid, sid])


class OpTomoTranspose(scipy.sparse.linalg.LinearOperator):
    """W.T of an OpTomo W: backprojection as the operator."""

    def __init__(self, parent):
        self.parent = parent
        super().__init__(np.float32, (parent.shape[1], parent.shape[0]))

    def _matvec(self, s):
        return self.parent.rmatvec(s)

    def _rmatvec(self, v):
        return self.parent._matvec(v)

    def _transpose(self):
        return self.parent

    _adjoint = _transpose

    def __mul__(self, s):
        if isinstance(s, torch.Tensor) or (isinstance(s, np.ndarray) and s.shape == self.parent.sshape):
            return self.parent.BP(s)
        return scipy.sparse.linalg.LinearOperator.__mul__(self, s)
