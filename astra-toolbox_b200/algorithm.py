"""astra.algorithm: reconstruction / projection algorithm objects.

Names and configuration keys follow the reference's algorithm factory
(include/astra/AlgorithmTypelist.h) and its config readers:
FP3D_CUDA (src/CudaForwardProjectionAlgorithm3D.cpp), BP3D_CUDA
(src/CudaBackProjectionAlgorithm3D.cpp), FDK_CUDA (src/CudaFDKAlgorithm3D.cpp),
SIRT3D_CUDA (src/CudaSirtAlgorithm3D.cpp), CGLS3D_CUDA
(src/CudaCglsAlgorithm3D.cpp), FP_CUDA, BP_CUDA, SIRT_CUDA, CGLS_CUDA, SART_CUDA,
FBP_CUDA (src/Cuda*Algorithm.cpp).  Every one of them runs in libb2tomo.
"""
import ctypes

import numpy as np
import torch

from . import _lib
from . import data as _d
from . import projector as _P
from ._lib import AstraError


def _opt(cfg):
    return dict(cfg.get('option', {}) or {})


def _filter_from_cfg(cfg, opt):
    """SFilterConfig from an algorithm config (getFilterConfigForAlgorithm,
    src/Filters.cpp:548-657): FilterType, FilterD, FilterParameter and, for
    the custom types, FilterSinogramId (a 2D sinogram data object), as
    options or as top-level keys."""
    def get(key, default=None):
        return opt.get(key, cfg.get(key, default))
    ftype = get('FilterType', 'ram-lak')
    code = _P.filter_code(ftype)
    custom = None
    if code >= _lib.FILTER_PROJECTION:
        fid = get('FilterSinogramId')
        if fid is None:
            raise AstraError(1, "FilterType %r needs FilterSinogramId" % (ftype,))
        custom = _d.lookup(fid, _d.DataObject).tensor.detach().cpu().numpy()
    return _P.FilterSpec(code, d=float(get('FilterD', 1.0)), parameter=float(get('FilterParameter', -1.0)),
                         custom=custom)


def _constraints(o):
    use_min = 'MinConstraint' in o or bool(o.get('UseMinConstraint', False))
    vmin = float(o.get('MinConstraint', o.get('MinConstraintValue', 0.0)))
    use_max = 'MaxConstraint' in o or bool(o.get('UseMaxConstraint', False))
    vmax = float(o.get('MaxConstraint', o.get('MaxConstraintValue', 255.0)))
    return use_min, vmin, use_max, vmax


class _Algorithm:
    def __init__(self, cfg):
        self.cfg = cfg
        self.opt = _opt(cfg)

    def _projector_options(self):
        """Options of the projector object, overridden by the algorithm's own."""
        o = {}
        if 'ProjectorId' in self.cfg:
            pr = _d.lookup(self.cfg['ProjectorId'])
            o.update(pr.options)
        for k in ('DetectorSuperSampling', 'VoxelSuperSampling', 'PixelSuperSampling', 'GPUIndex',
                  'ProjectionKernel'):
            if k in self.opt:
                o[k] = self.opt[k]
        return o

    def run(self, iterations=1):
        raise NotImplementedError

    def get_res_norm(self):
        raise AstraError(2, "%s has no residual norm" % self.cfg['type'])

    def close(self):
        pass


class _FP(_Algorithm):
    def __init__(self, cfg, is3d):
        super().__init__(cfg)
        self.vol = _d.lookup(cfg['VolumeDataId'], _d.DataObject)
        self.proj = _d.lookup(cfg['ProjectionDataId'], _d.DataObject)
        cls = _P.Projector3D if is3d else _P.Projector2D
        self.pr = cls(self.proj.geometry, self.vol.geometry, self._projector_options())
        self.is3d = is3d

    def run(self, iterations=1):
        if self.is3d and not (self.vol.tensor.is_cuda and self.proj.tensor.is_cuda):
            _P.fp3d_host(self.pr, self.vol.tensor, self.proj.tensor)
        else:
            self.pr.fp(self.vol.tensor, self.proj.tensor)
        self.proj.changed()


class _BP(_Algorithm):
    def __init__(self, cfg, is3d):
        super().__init__(cfg)
        self.vol = _d.lookup(cfg['ReconstructionDataId'], _d.DataObject)
        self.proj = _d.lookup(cfg['ProjectionDataId'], _d.DataObject)
        cls = _P.Projector3D if is3d else _P.Projector2D
        self.pr = cls(self.proj.geometry, self.vol.geometry, self._projector_options())
        self.is3d = is3d

    def run(self, iterations=1):
        if self.is3d and not (self.vol.tensor.is_cuda and self.proj.tensor.is_cuda):
            _P.bp3d_host(self.pr, self.proj.tensor, self.vol.tensor)
        else:
            self.pr.bp(self.proj.tensor, self.vol.tensor)
        self.vol.changed()


class _FDK(_Algorithm):
    def __init__(self, cfg):
        super().__init__(cfg)
        self.vol = _d.lookup(cfg['ReconstructionDataId'], _d.DataObject)
        self.proj = _d.lookup(cfg['ProjectionDataId'], _d.DataObject)
        self.pr = _P.Projector3D(self.proj.geometry, self.vol.geometry, self._projector_options())
        if self.pr.geom.kind != _lib.GEOM_CONE:
            raise AstraError(2, "FDK_CUDA needs a cone or cone_vec geometry")
        self.short = bool(self.opt.get('ShortScan', False))
        self.filter = _filter_from_cfg(cfg, self.opt)

    def run(self, iterations=1):
        if not (self.vol.tensor.is_cuda and self.proj.tensor.is_cuda):
            _P.fdk_host(self.pr, self.proj.tensor, self.vol.tensor, short_scan=self.short, filter_type=self.filter)
        else:
            _P.fdk(self.pr, self.proj.tensor, self.vol.tensor, short_scan=self.short, filter_type=self.filter)
        self.vol.changed()


class _Iterative(_Algorithm):
    """SIRT / CGLS through b2t_algo_* (2D or 3D)."""

    def __init__(self, cfg, kind, is3d):
        super().__init__(cfg)
        self.vol = _d.lookup(cfg['ReconstructionDataId'], _d.DataObject)
        self.proj = _d.lookup(cfg['ProjectionDataId'], _d.DataObject)
        po = self._projector_options()
        cls = _P.Projector3D if is3d else _P.Projector2D
        self.pr = cls(self.proj.geometry, self.vol.geometry, po)
        o = self.opt
        use_min, vmin, use_max, vmax = _constraints(o)
        self._keep = []

        def dev_ptr(key):
            if key not in o:
                return None
            obj = _d.lookup(o[key], _d.DataObject)
            # the library reads masks on the device: stage host-resident ones
            t = obj.tensor if obj.tensor.is_cuda else obj.tensor.to(torch.device('cuda', torch.cuda.current_device()))
            self._keep.extend([obj, t])
            return t.data_ptr()

        self.c_opt = _lib.AlgoOptions(float(o.get('Relaxation', 1.0)), int(use_min), vmin, int(use_max), vmax,
                                      dev_ptr('ReconstructionMaskId'), dev_ptr('SinogramMaskId'),
                                      dev_ptr('MinMaskId'), dev_ptr('MaxMaskId'))
        self.use_graph = int(bool(o.get('UseGraph', False)))
        self.handle = ctypes.c_void_p()
        if is3d:
            create = "b2t_algo_create3d_cyl" if self.pr.is_cyl else "b2t_algo_create3d"
            _lib.call(create, kind, ctypes.byref(self.pr.geom.c), ctypes.byref(self.pr.params()),
                      ctypes.byref(self.c_opt), ctypes.byref(self.handle))
        else:
            _lib.call("b2t_algo_create2d", kind, ctypes.byref(self.pr.geom.c), self.pr.det_ss, self.pr.pix_ss,
                      ctypes.byref(self.c_opt), ctypes.byref(self.handle))

    def _device_data(self):
        """(projection, volume) device tensors: host-resident data objects are
        staged on the GPU for the iterations (SIRT and CGLS need all of it on
        the device, as the reference's do)."""
        p, v = self.proj.tensor, self.vol.tensor
        dev = torch.device('cuda', torch.cuda.current_device())
        return (p if p.is_cuda else p.to(dev)), (v if v.is_cuda else v.to(dev))

    def run(self, iterations=1):
        p, v = self._device_data()
        with torch.cuda.device(v.device):
            _lib.call("b2t_algo_run", self.handle, p.data_ptr(), v.data_ptr(),
                      int(iterations), self.use_graph, _P.stream_handle(v.device))
        if not self.vol.tensor.is_cuda:
            self.vol.tensor.copy_(v.cpu())
        self.vol.changed()

    def get_res_norm(self):
        p, v = self._device_data()
        out = ctypes.c_double(0.0)
        with torch.cuda.device(v.device):
            _lib.call("b2t_algo_residual_norm", self.handle, p.data_ptr(), v.data_ptr(),
                      ctypes.byref(out), _P.stream_handle(v.device))
        return out.value

    def close(self):
        if self.handle:
            _lib.load().b2t_algo_destroy(self.handle)
            self.handle = ctypes.c_void_p()


class _SART(_Iterative):
    """SART_CUDA (src/CudaSartAlgorithm.cpp): one view per iteration.

    ProjectionOrder 'random' (the default, a uniform random permutation drawn
    once, as the reference's shuffle), 'sequential', or 'custom' with
    ProjectionOrderList; Relaxation is lambda."""

    def __init__(self, cfg):
        super().__init__(cfg, _lib.ALGO_SART, False)
        o = self.opt
        na = self.pr.proj_shape[0]
        kind = o.get('ProjectionOrder', 'random')
        if kind == 'sequential':
            order = None
        elif kind == 'random':
            order = np.random.default_rng().permutation(na)
        elif kind == 'custom':
            if 'ProjectionOrderList' not in o:
                raise AstraError(1, "SART_CUDA: ProjectionOrder 'custom' needs ProjectionOrderList")
            order = np.asarray(o['ProjectionOrderList']).ravel()
        else:
            raise AstraError(1, "SART_CUDA: Unknown ProjectionOrder %r" % (kind,))
        if order is not None:
            arr = np.ascontiguousarray(order, dtype=np.int32)
            _lib.call("b2t_algo_set_projection_order", self.handle, arr.ctypes.data, int(arr.size))


class _FBP2D(_Algorithm):
    def __init__(self, cfg):
        super().__init__(cfg)
        self.vol = _d.lookup(cfg['ReconstructionDataId'], _d.DataObject)
        self.proj = _d.lookup(cfg['ProjectionDataId'], _d.DataObject)
        self.pr = _P.Projector2D(self.proj.geometry, self.vol.geometry, self._projector_options())
        self.short = bool(self.opt.get('ShortScan', False))
        self.filter = _filter_from_cfg(cfg, self.opt)

    def run(self, iterations=1):
        _P.fbp2d(self.pr, self.proj.tensor, self.vol.tensor, short_scan=self.short, filter_type=self.filter)
        self.vol.changed()


_FACTORY = {
    'FP3D_CUDA': lambda c: _FP(c, True),
    'BP3D_CUDA': lambda c: _BP(c, True),
    'FDK_CUDA': _FDK,
    'SIRT3D_CUDA': lambda c: _Iterative(c, _lib.ALGO_SIRT, True),
    'CGLS3D_CUDA': lambda c: _Iterative(c, _lib.ALGO_CGLS, True),
    'FP_CUDA': lambda c: _FP(c, False),
    'BP_CUDA': lambda c: _BP(c, False),
    'SIRT_CUDA': lambda c: _Iterative(c, _lib.ALGO_SIRT, False),
    'CGLS_CUDA': lambda c: _Iterative(c, _lib.ALGO_CGLS, False),
    'SART_CUDA': _SART,
    'FBP_CUDA': _FBP2D,
}


def astra_dict(intype):
    """An algorithm configuration dictionary (python/astra/functions.py astra_dict)."""
    if intype not in _FACTORY:
        raise AstraError(2, "Unknown algorithm type %r" % (intype,))
    return {'type': intype, 'option': {}}


def create(cfg):
    t = cfg.get('type')
    if t not in _FACTORY:
        raise AstraError(2, "Unknown algorithm type %r" % (t,))
    return _d.register(_FACTORY[t](cfg))


def run(i, iterations=1):
    _d.lookup(i, _Algorithm).run(iterations)


def get_res_norm(i):
    return _d.lookup(i, _Algorithm).get_res_norm()


def abort(i):
    a = _d.lookup(i, _Algorithm)
    if isinstance(a, _Iterative) and a.handle:
        _lib.load().b2t_algo_abort(a.handle)


def delete(ids):
    for i in (ids if isinstance(ids, (list, tuple)) else [ids]):
        try:
            _d.lookup(i, _Algorithm).close()
        except AstraError:
            pass
        _d.remove(i)


def clear():
    for i in _d.ids_of(_Algorithm):
        delete(i)
