"""The 'cuda3d' and 'cuda' projector objects and the direct FP/BP calls.

Mirrors the reference's CCudaProjector3D / CCudaProjector2D options
(src/CudaProjector3D.cpp:94-118, src/CudaProjector2D.cpp:84-100) and
astra.experimental.direct_FP3D / direct_BP3D
(python/astra/experimental.pyx:172-227): data are torch tensors on a CUDA
device (or numpy arrays, which are copied to the device and back), all work is
done by libb2tomo kernels on the current torch stream.
"""
import ctypes

import numpy as np
import torch

from . import _lib
from ._lib import AstraError
from .geometry import Geometry2D, Geometry3D, is_3d_vol

_KERNELS = {
    'default': _lib.KER_DEFAULT, 'sum_square_weights': _lib.KER_SUM_SQUARE_WEIGHTS,
    '2d_weighting': _lib.KER_2D_WEIGHTING, 'matched_bp': _lib.KER_MATCHED_BP,
    'fdk_weighting': _lib.KER_FDK_WEIGHTING,
}

_DTYPES = {torch.float32: _lib.F32, torch.float16: _lib.F16, torch.bfloat16: _lib.BF16}


def stream_handle(device=None):
    """cudaStream_t of torch's current stream on device, as an int."""
    return torch.cuda.current_stream(device).cuda_stream


def _check_tensor(t, shape, name, device=None):
    if not isinstance(t, torch.Tensor):
        raise AstraError(1, "%s must be a torch tensor" % name)
    if not t.is_cuda:
        raise AstraError(1, "%s must be on a CUDA device" % name)
    if tuple(t.shape) != tuple(shape):
        raise AstraError(1, "%s has shape %s, geometry needs %s" % (name, tuple(t.shape), tuple(shape)))
    if t.dtype not in _DTYPES:
        raise AstraError(1, "%s must be float32, float16 or bfloat16" % name)
    if not t.is_contiguous():
        raise AstraError(1, "%s must be contiguous" % name)
    if device is not None and t.device != device:
        raise AstraError(1, "%s is on %s, expected %s" % (name, t.device, device))


class Projector3D:
    """A 'cuda3d' projector: geometry plus projection options."""

    def __init__(self, proj_geom, vol_geom, options=None):
        options = dict(options or {})
        self.options = options
        self.proj_geom = proj_geom
        self.vol_geom = vol_geom
        self.geom = Geometry3D(vol_geom, proj_geom)
        kname = options.get('ProjectionKernel', 'default')
        if kname not in _KERNELS:
            raise AstraError(1, "Unknown ProjectionKernel %r" % kname)
        self.kernel = _KERNELS[kname]
        self.det_ss = int(options.get('DetectorSuperSampling', 1))
        self.vox_ss = int(options.get('VoxelSuperSampling', 1))
        self.gpu_index = int(options.get('GPUIndex', -1))
        self.vol_shape = self.geom.vol_shape
        self.proj_shape = self.geom.proj_shape

    def params(self, output_scale=1.0, kernel=None):
        return _lib.Params3D(self.det_ss, self.vox_ss, float(output_scale),
                             self.kernel if kernel is None else kernel)

    def device(self):
        if self.gpu_index >= 0:
            return torch.device('cuda', self.gpu_index)
        return torch.device('cuda', torch.cuda.current_device())

    def fp(self, vol, proj, mode=_lib.MODE_SET, output_scale=1.0, kernel=None):
        """proj (=|+=) A vol on torch tensors."""
        _check_tensor(vol, self.vol_shape, "volume")
        _check_tensor(proj, self.proj_shape, "projection data", vol.device)
        if vol.dtype != proj.dtype:
            raise AstraError(1, "volume and projection data must have the same dtype")
        p = self.params(output_scale, kernel)
        with torch.cuda.device(vol.device):
            if self.is_cyl:
                self._cyl_f32(vol)
                _lib.call("b2t_fp3d_cyl", ctypes.byref(self.geom.c), ctypes.byref(p), vol.data_ptr(), 0,
                          proj.data_ptr(), 0, mode, stream_handle(vol.device))
            else:
                _lib.call("b2t_fp3d", ctypes.byref(self.geom.c), ctypes.byref(p), vol.data_ptr(), 0,
                          proj.data_ptr(), 0, _DTYPES[vol.dtype], mode, stream_handle(vol.device))
        return proj

    @property
    def is_cyl(self):
        return self.geom.kind == _lib.GEOM_CYLCONE

    @staticmethod
    def _cyl_f32(t):
        if t.dtype != torch.float32:
            raise AstraError(1, "cyl_cone_vec projectors take float32 data")

    def autotune(self, vol, proj):
        """Time the forward projector's launch shapes on these buffers and keep
        the fastest for this problem class (b2t_autotune_fp3d); proj is
        overwritten with A vol.  Returns the chosen views per CTA."""
        _check_tensor(vol, self.vol_shape, "volume")
        _check_tensor(proj, self.proj_shape, "projection data", vol.device)
        if self.is_cyl:
            raise AstraError(3, "autotune: the cyl_cone_vec projector has a single launch shape")
        p = self.params()
        vpc = ctypes.c_int32(0)
        with torch.cuda.device(vol.device):
            _lib.call("b2t_autotune_fp3d", ctypes.byref(self.geom.c), ctypes.byref(p), vol.data_ptr(), 0,
                      proj.data_ptr(), 0, _DTYPES[vol.dtype], stream_handle(vol.device), ctypes.byref(vpc))
        return vpc.value

    def autotune_bp(self, proj, vol):
        """Time the TMA backprojector's launch shapes on these buffers and keep
        the fastest for this problem class (b2t_autotune_bp3d); vol is
        overwritten with B proj.  Returns the chosen voxels per thread."""
        _check_tensor(vol, self.vol_shape, "volume")
        _check_tensor(proj, self.proj_shape, "projection data", vol.device)
        if self.is_cyl:
            raise AstraError(3, "autotune_bp: the cyl_cone_vec projector has a single launch shape")
        p = self.params()
        vpt = ctypes.c_int32(0)
        with torch.cuda.device(vol.device):
            _lib.call("b2t_autotune_bp3d", ctypes.byref(self.geom.c), ctypes.byref(p), proj.data_ptr(), 0,
                      vol.data_ptr(), 0, _DTYPES[vol.dtype], stream_handle(vol.device), ctypes.byref(vpt))
        return vpt.value

    def bp(self, proj, vol, mode=_lib.MODE_SET, output_scale=1.0, kernel=None):
        """vol (=|+=) B proj on torch tensors (B = ASTRA's BP, or A^T for matched_bp)."""
        _check_tensor(vol, self.vol_shape, "volume")
        _check_tensor(proj, self.proj_shape, "projection data", vol.device)
        if vol.dtype != proj.dtype:
            raise AstraError(1, "volume and projection data must have the same dtype")
        p = self.params(output_scale, kernel)
        with torch.cuda.device(vol.device):
            if self.is_cyl:
                self._cyl_f32(vol)
                _lib.call("b2t_bp3d_cyl", ctypes.byref(self.geom.c), ctypes.byref(p), proj.data_ptr(), 0,
                          vol.data_ptr(), 0, mode, stream_handle(vol.device))
            else:
                _lib.call("b2t_bp3d", ctypes.byref(self.geom.c), ctypes.byref(p), proj.data_ptr(), 0,
                          vol.data_ptr(), 0, _DTYPES[vol.dtype], mode, stream_handle(vol.device))
        return vol


class Projector2D:
    """A 'cuda' projector: 2D geometry plus DetectorSuperSampling /
    PixelSuperSampling (src/CudaProjector2D.cpp:84-100)."""

    def __init__(self, proj_geom, vol_geom, options=None):
        options = dict(options or {})
        self.options = options
        self.proj_geom = proj_geom
        self.vol_geom = vol_geom
        self.geom = Geometry2D(vol_geom, proj_geom)
        self.det_ss = int(options.get('DetectorSuperSampling', 1))
        self.pix_ss = int(options.get('PixelSuperSampling', 1))
        self.gpu_index = int(options.get('GPUIndex', -1))
        self.vol_shape = self.geom.vol_shape
        self.proj_shape = self.geom.proj_shape

    def device(self):
        if self.gpu_index >= 0:
            return torch.device('cuda', self.gpu_index)
        return torch.device('cuda', torch.cuda.current_device())

    def fp(self, vol, sino, mode=_lib.MODE_SET):
        _check_tensor(vol, self.vol_shape, "volume")
        _check_tensor(sino, self.proj_shape, "sinogram", vol.device)
        if vol.dtype != torch.float32 or sino.dtype != torch.float32:
            raise AstraError(1, "2D data must be float32")
        with torch.cuda.device(vol.device):
            _lib.call("b2t_fp2d", ctypes.byref(self.geom.c), self.det_ss, vol.data_ptr(), 0, sino.data_ptr(), 0,
                      mode, stream_handle(vol.device))
        return sino

    def bp(self, sino, vol, mode=_lib.MODE_SET, fbp_weight=False):
        _check_tensor(vol, self.vol_shape, "volume")
        _check_tensor(sino, self.proj_shape, "sinogram", vol.device)
        if vol.dtype != torch.float32 or sino.dtype != torch.float32:
            raise AstraError(1, "2D data must be float32")
        with torch.cuda.device(vol.device):
            _lib.call("b2t_bp2d", ctypes.byref(self.geom.c), self.pix_ss, int(bool(fbp_weight)), sino.data_ptr(), 0,
                      vol.data_ptr(), 0, mode, stream_handle(vol.device))
        return vol


def dlpack_tensor(x):
    """(torch tensor sharing x's memory, True) for a DLPack object or capsule
    other than a torch tensor or numpy array; (None, False) otherwise.

    The reference takes DLPack data without a stream (its getDLPackCapsule,
    python/astra/utils.pyx:237-260, leaves the stream argument open).  Here the
    exchange follows the DLPack protocol: torch.from_dlpack passes the current
    torch stream of the data's device to __dlpack__, so the producer orders its
    pending work before the kernels that will read or write the array."""
    if isinstance(x, (torch.Tensor, np.ndarray)):
        return None, False
    is_capsule = type(x).__name__ == 'PyCapsule'
    if not (hasattr(x, '__dlpack__') or is_capsule):
        return None, False
    try:
        return torch.from_dlpack(x), True
    except Exception as e:  # unsupported device, dtype or layout
        raise AstraError(1, "cannot use the DLPack data: %s" % (e,))


def as_device_tensor(x, device, dtype=None):
    """(tensor on device, copy_back) for a numpy array, a torch tensor or any
    DLPack object (CUDA data in place; host data copied)."""
    t, _ = dlpack_tensor(x)
    if t is not None:
        x = t
    if isinstance(x, np.ndarray):
        if x.dtype != np.float32:
            raise AstraError(1, "numpy data must be float32")
        return torch.from_numpy(np.ascontiguousarray(x)).to(device), True
    if isinstance(x, torch.Tensor):
        if x.is_cuda:
            return x, False
        return x.to(device), True
    raise AstraError(1, "data must be a numpy array, a torch tensor or a DLPack object")


def _finish_foreign(outputs, device):
    """After writing into arrays that came through DLPack from another
    library: synchronise the stream, so the producer's own streams see the
    results (DLPack orders the hand-over, not the hand-back)."""
    if any(dlpack_tensor(o)[1] for o in outputs):
        torch.cuda.current_stream(device).synchronize()


def _write_back(x, t):
    """Copy a device result into the host object it came from."""
    if isinstance(x, np.ndarray):
        x[...] = t.cpu().numpy()
        return
    d, _ = dlpack_tensor(x)
    (d if d is not None else x).copy_(t.cpu())


def fp3d(projector, vol, proj, mode=_lib.MODE_SET):
    """direct_FP3D semantics on numpy arrays or torch tensors (written in place)."""
    dev = projector.device()
    tv, _ = as_device_tensor(vol, dev)
    tp, back = as_device_tensor(proj, dev)
    projector.fp(tv, tp, mode=mode)
    if back:
        _write_back(proj, tp)
    _finish_foreign([proj], dev)
    return proj


def bp3d(projector, vol, proj, mode=_lib.MODE_SET):
    """direct_BP3D semantics on numpy arrays or torch tensors (vol written in place)."""
    dev = projector.device()
    tp, _ = as_device_tensor(proj, dev)
    tv, back = as_device_tensor(vol, dev)
    projector.bp(tp, tv, mode=mode)
    if back:
        _write_back(vol, tv)
    _finish_foreign([vol], dev)
    return vol


def filter_code(name):
    """FilterType option -> filter code (the reference's names, src/Filters.cpp:
    508-532, case-insensitive; 'ramlak' is accepted for 'ram-lak')."""
    key = (name or 'ram-lak').lower()
    if key == 'ramlak':
        key = 'ram-lak'
    if key not in _lib.FILTER_NAMES:
        raise AstraError(2, "Failed to convert %r into a filter" % (name,))
    return _lib.FILTER_NAMES.index(key)


class FilterSpec:
    """A filter for FDK / FBP / row filtering: SFilterConfig's fields
    (include/astra/Filters.h:70-82).  `custom` is a 1D or 2D array for the
    projection / sinogram / rprojection / rsinogram types."""

    def __init__(self, filter_type='ram-lak', d=1.0, parameter=-1.0, custom=None):
        self.type = filter_code(filter_type) if isinstance(filter_type, str) else int(filter_type)
        self.d = float(d)
        self.parameter = float(parameter)
        self.custom = None
        if custom is not None:
            c = np.ascontiguousarray(np.asarray(custom, dtype=np.float32))
            self.custom = c.reshape(1, -1) if c.ndim == 1 else c

    def c(self):
        """The ctypes b2t_filter_config (valid while this object lives)."""
        cfg = _lib.FilterConfig(self.type, self.d, self.parameter, None, 0, 0)
        if self.custom is not None:
            cfg.custom = self.custom.ctypes.data
            cfg.custom_height, cfg.custom_width = self.custom.shape
        return cfg


def _filter_spec(filter_type):
    return filter_type if isinstance(filter_type, FilterSpec) else FilterSpec(filter_type)


def filter_taps(filter_type, n, n_views=1):
    """The filter's exact spatial taps (b2t_filter_taps): array (sets, 2n-1),
    tap of offset d at column d + n - 1."""
    spec = _filter_spec(filter_type)
    cfg = spec.c()
    count = ctypes.c_size_t(0)
    _lib.call("b2t_filter_taps", ctypes.byref(cfg), int(n), int(n_views), None, ctypes.byref(count))
    out = np.zeros(count.value, dtype=np.float32)
    _lib.call("b2t_filter_taps", ctypes.byref(cfg), int(n), int(n_views), out.ctypes.data, ctypes.byref(count))
    return out.reshape(-1, 2 * int(n) - 1)


# ---------------------------------------------------------------------------
# streamed calls on host-resident data (b2t_*_host)
# ---------------------------------------------------------------------------

def _host_f32(t):
    if t.is_cuda:
        return t.cpu().contiguous(), True
    if t.dtype != torch.float32 or not t.is_contiguous():
        raise AstraError(1, "host data must be contiguous float32")
    return t, False


def _stream(fn, projector, inp, out, extra_before, extra_after, mode):
    """Run a b2t_*_host call: inputs and outputs as CPU tensors (device
    tensors are staged through host memory)."""
    from . import gpu as _gpu
    if projector.is_cyl:
        raise AstraError(3, "streamed projection covers the flat-panel geometries; cyl_cone_vec data must fit the GPU")
    hi, _ = _host_f32(inp)
    ho, staged = _host_f32(out)
    cfg = _gpu.stream_config()
    _lib.call(fn, ctypes.byref(projector.geom.c), *extra_before, hi.data_ptr(), ho.data_ptr(), mode, *extra_after,
              ctypes.byref(cfg))
    if staged:
        out.copy_(ho)
    return out


def fp3d_host(projector, vol, proj, mode=_lib.MODE_SET):
    """proj (=|+=) A vol, streamed through the GPUs (b2t_fp3d_host)."""
    return _stream("b2t_fp3d_host", projector, vol, proj, [ctypes.byref(projector.params())], [], mode)


def bp3d_host(projector, proj, vol, mode=_lib.MODE_SET):
    """vol (=|+=) B proj, streamed through the GPUs (b2t_bp3d_host)."""
    return _stream("b2t_bp3d_host", projector, proj, vol, [ctypes.byref(projector.params())], [], mode)


def fdk_host(projector, proj, vol, short_scan=False, filter_type='ram-lak', output_scale=1.0, mode=_lib.MODE_SET):
    """FDK streamed through the GPUs (b2t_fdk_host)."""
    _no_cyl(projector, "FDK")
    cfg = _filter_spec(filter_type).c()
    return _stream("b2t_fdk_host", projector, proj, vol,
                   [ctypes.byref(cfg), int(bool(short_scan)), ctypes.c_float(output_scale)], [], mode)


def stream_plan(projector, op):
    """(z-slab thickness, angle block size) of a streamed FP ('fp'), BP
    ('bp') or FDK ('fdk') under the current GPU settings."""
    from . import gpu as _gpu
    cfg = _gpu.stream_config()
    slab, block = ctypes.c_uint32(0), ctypes.c_uint32(0)
    _lib.call("b2t_stream_plan", {'fp': 0, 'bp': 1, 'fdk': 2}[op], ctypes.byref(projector.geom.c),
              ctypes.byref(cfg), ctypes.byref(slab), ctypes.byref(block))
    return slab.value, block.value


def _no_cyl(projector, what):
    # FDK needs a flat-panel cone geometry (cuda/3d/fdk.cu:415-478)
    if getattr(projector, 'is_cyl', False):
        raise AstraError(3, "%s needs a flat-panel cone geometry, not cyl_cone_vec" % what)


def fdk(projector, proj, vol, short_scan=False, filter_type='ram-lak', output_scale=1.0, mode=_lib.MODE_SET):
    """FDK of proj into vol (torch CUDA tensors); proj is not modified."""
    _no_cyl(projector, "FDK")
    _check_tensor(vol, projector.vol_shape, "volume")
    _check_tensor(proj, projector.proj_shape, "projection data", vol.device)
    if vol.dtype != proj.dtype:
        raise AstraError(1, "volume and projection data must have the same dtype")
    with torch.cuda.device(vol.device):
        spec = _filter_spec(filter_type)
        cfg = spec.c()
        _lib.call("b2t_fdk", ctypes.byref(projector.geom.c), ctypes.byref(cfg), int(bool(short_scan)),
                  float(output_scale), proj.data_ptr(), 0, vol.data_ptr(), 0, _DTYPES[vol.dtype], mode,
                  stream_handle(vol.device))
    return vol


def fbp2d(projector, sino, vol, short_scan=False, filter_type='ram-lak', mode=_lib.MODE_SET):
    """2D FBP of sino into vol (torch CUDA float32); sino is not modified."""
    _check_tensor(vol, projector.vol_shape, "volume")
    _check_tensor(sino, projector.proj_shape, "sinogram", vol.device)
    with torch.cuda.device(vol.device):
        spec = _filter_spec(filter_type)
        cfg = spec.c()
        _lib.call("b2t_fbp2d", ctypes.byref(projector.geom.c), ctypes.byref(cfg), int(bool(short_scan)),
                  sino.data_ptr(), 0, vol.data_ptr(), 0, mode, stream_handle(vol.device))
    return vol


# ---------------------------------------------------------------------------
# astra.projector: registry of 2D 'cuda' projectors (python/astra/projector.py)
# ---------------------------------------------------------------------------

def create(cfg):
    """Create a projector from a configuration dict; 'cuda' (2D) or 'cuda3d'."""
    from . import data as _d
    t = cfg.get('type')
    opts = dict(cfg.get('options', cfg.get('option', {})) or {})
    if t == 'cuda':
        return _d.register(Projector2D(cfg['ProjectionGeometry'], cfg['VolumeGeometry'], opts))
    if t == 'cuda3d':
        return _d.register(Projector3D(cfg['ProjectionGeometry'], cfg['VolumeGeometry'], opts))
    raise AstraError(2, "Projector type %r is not available (cuda and cuda3d are)" % (t,))


def delete(ids):
    from . import data as _d
    for i in (ids if isinstance(ids, (list, tuple)) else [ids]):
        _d.remove(i)


def clear():
    from . import data as _d
    for i in _d.ids_of(Projector2D) + _d.ids_of(Projector3D):
        _d.remove(i)


def lookup_projector(i):
    from . import data as _d
    pr = _d.lookup(i)
    if not isinstance(pr, (Projector2D, Projector3D)):
        raise AstraError(1, "Not a projector id: %r" % (i,))
    return pr


def projection_geometry(i):
    from . import data as _d
    return _d.lookup(i).proj_geom


def volume_geometry(i):
    from . import data as _d
    return _d.lookup(i).vol_geom


def fdk_weight_filter(projector, proj, short_scan=False, filter_type='ram-lak'):
    """FDK pre-weighting and filtering of proj in place."""
    _no_cyl(projector, "FDK")
    _check_tensor(proj, projector.proj_shape, "projection data")
    with torch.cuda.device(proj.device):
        spec = _filter_spec(filter_type)
        cfg = spec.c()
        _lib.call("b2t_fdk_weight_filter", ctypes.byref(projector.geom.c), ctypes.byref(cfg),
                  int(bool(short_scan)), proj.data_ptr(), 0, _DTYPES[proj.dtype], stream_handle(proj.device))
    return proj
