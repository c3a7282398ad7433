"""Batched problems: many independent 'cuda' 2D problems (parallel and fan,
any sizes and angle counts) projected or reconstructed together, and many
3D problems (parallel3d / parallel3d_vec / cone / cone_vec) projected
together, one persistent GPU launch per operation (b2t_batch2d_* and
b2t_batch3d_* in libb2tomo).

The reference has no batched form; a user loops over problems, creating a
projector and running FP_CUDA / BP_CUDA / SIRT_CUDA for each
(src/CudaForwardProjectionAlgorithm.cpp, src/CudaSirtAlgorithm.cpp).  Here
the problems' volumes and sinograms live in two packed float32 CUDA tensors;
`vol_views` / `sino_views` give per-problem views into them.
"""
import ctypes

import numpy as np
import torch

from . import _lib
from ._lib import AstraError
from .geometry import Geometry2D, Geometry3D
from .projector import stream_handle


class Batch2D:
    """A planned batch.  `problems` is a list of (proj_geom, vol_geom) or
    (proj_geom, vol_geom, options) with the 'cuda' projector options
    DetectorSuperSampling / PixelSuperSampling."""

    def __init__(self, problems, device=None):
        self.device = torch.device(device) if device is not None else torch.device('cuda', torch.cuda.current_device())
        self.geoms = []
        n = len(problems)
        if n == 0:
            raise AstraError(1, "a batch needs at least one problem")
        arr = (_lib.Problem2D * n)()
        for i, pb in enumerate(problems):
            pg, vg = pb[0], pb[1]
            opts = dict(pb[2]) if len(pb) > 2 and pb[2] else {}
            g = Geometry2D(vg, pg)
            self.geoms.append(g)
            arr[i].geom = g.c
            arr[i].det_supersample = int(opts.get('DetectorSuperSampling', 1))
            arr[i].pixel_supersample = int(opts.get('PixelSuperSampling', 1))
        self.handle = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            _lib.call("b2t_batch2d_create", arr, n, ctypes.byref(self.handle))
        vo = (ctypes.c_uint64 * n)()
        so = (ctypes.c_uint64 * n)()
        vt = ctypes.c_uint64(0)
        st = ctypes.c_uint64(0)
        _lib.call("b2t_batch2d_layout", self.handle, vo, so, ctypes.byref(vt), ctypes.byref(st))
        self.vol_offsets = [int(x) for x in vo]
        self.sino_offsets = [int(x) for x in so]
        self.vol_total = int(vt.value)
        self.sino_total = int(st.value)
        self.vol_shapes = [g.vol_shape for g in self.geoms]
        self.proj_shapes = [g.proj_shape for g in self.geoms]

    def __len__(self):
        return len(self.geoms)

    # packed buffers and per-problem views -------------------------------------
    def empty_vols(self):
        return torch.zeros(self.vol_total, dtype=torch.float32, device=self.device)

    def empty_sinos(self):
        return torch.zeros(self.sino_total, dtype=torch.float32, device=self.device)

    def vol_views(self, packed):
        return [packed[o:o + int(np.prod(sh))].view(sh) for o, sh in zip(self.vol_offsets, self.vol_shapes)]

    def sino_views(self, packed):
        return [packed[o:o + int(np.prod(sh))].view(sh) for o, sh in zip(self.sino_offsets, self.proj_shapes)]

    def pack_vols(self, vols):
        out = self.empty_vols()
        for v, dst in zip(vols, self.vol_views(out)):
            dst.copy_(torch.as_tensor(v, dtype=torch.float32))
        return out

    def pack_sinos(self, sinos):
        out = self.empty_sinos()
        for v, dst in zip(sinos, self.sino_views(out)):
            dst.copy_(torch.as_tensor(v, dtype=torch.float32))
        return out

    def _check(self, t, n, what):
        if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.float32 and t.is_contiguous()
                and t.numel() == n):
            raise AstraError(1, "%s must be a contiguous float32 CUDA tensor of %d elements" % (what, n))

    # operations ----------------------------------------------------------------
    def fp(self, vols, sinos=None, mode=_lib.MODE_SET):
        """sinos (=|+=) A vols for every problem; returns sinos."""
        self._check(vols, self.vol_total, "packed volumes")
        sinos = self.empty_sinos() if sinos is None else sinos
        self._check(sinos, self.sino_total, "packed sinograms")
        with torch.cuda.device(self.device):
            _lib.call("b2t_batch2d_fp", self.handle, vols.data_ptr(), sinos.data_ptr(), mode,
                      stream_handle(self.device))
        return sinos

    def bp(self, sinos, vols=None, mode=_lib.MODE_SET):
        """vols (=|+=) backprojection of sinos for every problem; returns vols."""
        self._check(sinos, self.sino_total, "packed sinograms")
        vols = self.empty_vols() if vols is None else vols
        self._check(vols, self.vol_total, "packed volumes")
        with torch.cuda.device(self.device):
            _lib.call("b2t_batch2d_bp", self.handle, sinos.data_ptr(), vols.data_ptr(), mode,
                      stream_handle(self.device))
        return vols

    def sirt(self, sinos, vols, iterations, use_graph=True, relaxation=1.0, min_constraint=None,
             max_constraint=None):
        """SIRT_CUDA on every problem at once; vols is updated in place.
        Returns the batch's residual norm ||b - A x|| over all problems."""
        return self._iterate(_lib.ALGO_SIRT, sinos, vols, iterations, use_graph, relaxation, min_constraint,
                             max_constraint)

    def cgls(self, sinos, vols, iterations, use_graph=True):
        """CGLS_CUDA on every problem at once (per-problem step sizes); vols
        is updated in place.  Returns the batch's residual norm."""
        return self._iterate(_lib.ALGO_CGLS, sinos, vols, iterations, use_graph, 1.0, None, None)

    def _iterate(self, kind, sinos, vols, iterations, use_graph, relaxation, min_constraint, max_constraint):
        self._check(sinos, self.sino_total, "packed sinograms")
        self._check(vols, self.vol_total, "packed volumes")
        opt = _lib.AlgoOptions(float(relaxation), int(min_constraint is not None),
                               float(min_constraint or 0.0), int(max_constraint is not None),
                               float(max_constraint if max_constraint is not None else 0.0), None, None, None, None)
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            _lib.call("b2t_algo_create_batch2d", kind, self.handle, ctypes.byref(opt), ctypes.byref(h))
            try:
                _lib.call("b2t_algo_run", h, sinos.data_ptr(), vols.data_ptr(), int(iterations), int(bool(use_graph)),
                          stream_handle(self.device))
                res = ctypes.c_double(0.0)
                _lib.call("b2t_algo_residual_norm", h, sinos.data_ptr(), vols.data_ptr(), ctypes.byref(res),
                          stream_handle(self.device))
            finally:
                _lib.load().b2t_algo_destroy(h)
        return res.value

    def close(self):
        if self.handle:
            _lib.load().b2t_batch2d_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch3D:
    """A planned batch of 3D problems.  `problems` is a list of (proj_geom,
    vol_geom) or (proj_geom, vol_geom, options) with the 'cuda3d' projector
    option DetectorSuperSampling; FP32 data, the default BP weighting.
    Volumes (z, y, x) and projections (v, angle, u) live in two packed float32
    CUDA tensors; `vol_views` / `proj_views` give per-problem views into
    them.  A batch of identical problems packs them back to back, so a
    tensor with a leading batch dimension is a packed buffer as it is."""

    def __init__(self, problems, device=None):
        self.device = torch.device(device) if device is not None else torch.device('cuda', torch.cuda.current_device())
        n = len(problems)
        if n == 0:
            raise AstraError(1, "a batch needs at least one problem")
        self.geoms = []
        arr = (_lib.Problem3D * n)()
        for i, pb in enumerate(problems):
            pg, vg = pb[0], pb[1]
            opts = dict(pb[2]) if len(pb) > 2 and pb[2] else {}
            if pg['type'] == 'cyl_cone_vec':
                raise AstraError(2, "a 3D batch takes parallel3d(_vec) and cone(_vec) geometries")
            g = Geometry3D(vg, pg)
            self.geoms.append(g)
            arr[i].geom = g.c
            arr[i].det_supersample = int(opts.get('DetectorSuperSampling', 1))
            arr[i].output_scale = 1.0
        self.handle = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            _lib.call("b2t_batch3d_create", arr, n, ctypes.byref(self.handle))
        vo = (ctypes.c_uint64 * n)()
        po = (ctypes.c_uint64 * n)()
        vt = ctypes.c_uint64(0)
        pt = ctypes.c_uint64(0)
        _lib.call("b2t_batch3d_layout", self.handle, vo, po, ctypes.byref(vt), ctypes.byref(pt))
        self.vol_offsets = [int(x) for x in vo]
        self.proj_offsets = [int(x) for x in po]
        self.vol_total = int(vt.value)
        self.proj_total = int(pt.value)
        self.vol_shapes = [g.vol_shape for g in self.geoms]
        self.proj_shapes = [g.proj_shape for g in self.geoms]

    def __len__(self):
        return len(self.geoms)

    def empty_vols(self):
        return torch.zeros(self.vol_total, dtype=torch.float32, device=self.device)

    def empty_projs(self):
        return torch.zeros(self.proj_total, dtype=torch.float32, device=self.device)

    def vol_views(self, packed):
        return [packed.view(-1)[o:o + int(np.prod(sh))].view(sh) for o, sh in zip(self.vol_offsets, self.vol_shapes)]

    def proj_views(self, packed):
        return [packed.view(-1)[o:o + int(np.prod(sh))].view(sh) for o, sh in zip(self.proj_offsets,
                                                                                   self.proj_shapes)]

    def pack_vols(self, vols):
        out = self.empty_vols()
        for v, dst in zip(vols, self.vol_views(out)):
            dst.copy_(torch.as_tensor(v, dtype=torch.float32))
        return out

    def pack_projs(self, projs):
        out = self.empty_projs()
        for v, dst in zip(projs, self.proj_views(out)):
            dst.copy_(torch.as_tensor(v, dtype=torch.float32))
        return out

    def _check(self, t, n, what):
        if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.float32 and t.is_contiguous()
                and t.numel() == n):
            raise AstraError(1, "%s must be a contiguous float32 CUDA tensor of %d elements" % (what, n))

    def fp(self, vols, projs=None, mode=_lib.MODE_SET):
        """projs (=|+=) FP of vols for every problem; returns projs."""
        self._check(vols, self.vol_total, "packed volumes")
        projs = self.empty_projs() if projs is None else projs
        self._check(projs, self.proj_total, "packed projections")
        with torch.cuda.device(self.device):
            _lib.call("b2t_batch3d_fp", self.handle, vols.data_ptr(), projs.data_ptr(), mode,
                      stream_handle(self.device))
        return projs

    def bp(self, projs, vols=None, mode=_lib.MODE_SET, matched=False):
        """vols (=|+=) BP of projs for every problem (matched: the exact
        adjoint A^T of fp); returns vols."""
        self._check(projs, self.proj_total, "packed projections")
        vols = self.empty_vols() if vols is None else vols
        self._check(vols, self.vol_total, "packed volumes")
        with torch.cuda.device(self.device):
            _lib.call("b2t_batch3d_matched_bp" if matched else "b2t_batch3d_bp", self.handle, projs.data_ptr(),
                      vols.data_ptr(), mode, stream_handle(self.device))
        return vols

    def close(self):
        if self.handle:
            _lib.load().b2t_batch3d_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
