"""ctypes wrapper of oracle/_ref/libastra_ref.so (the reference built from its
own sources by oracle/ref.mk, plus oracle/ref_wrap.cu).

TEST INFRASTRUCTURE ONLY (tests/, and the reference legs of bench.py).
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(_HERE, "_ref", "libastra_ref.so")
_lib = None
_P = ctypes.c_void_p
_I = ctypes.c_int
_F = ctypes.c_float

GEOM3D_TYPES = {'parallel3d': 0, 'cone': 1, 'parallel3d_vec': 2, 'cone_vec': 3, 'cyl_cone_vec': 4}
GEOM2D_TYPES = {'parallel': 0, 'fanflat': 1, 'parallel_vec': 2, 'fanflat_vec': 3}


def available():
    return os.path.exists(LIB)


# The reference built with its cuda/3d projectors replaced by libb2tomo
# (oracle/ref_shim.mk): the same entry points, the reference's own host code
# (CompositeGeometryManager, FDK, algorithm objects) running on the library.
LIB_SHIM = os.path.join(_HERE, "_ref", "libastra_ref_shim.so")
_shim = None
_use_shim = False


def shim_available():
    return os.path.exists(LIB_SHIM)


class use_shim:
    """with use_shim(): every function of this module calls the shim build."""

    def __enter__(self):
        global _use_shim
        self._prev = _use_shim
        _use_shim = True
        return self

    def __exit__(self, *exc):
        global _use_shim
        _use_shim = self._prev
        return False


def lib():
    global _lib, _shim
    if _use_shim:
        if _shim is None:
            _shim = _declare(ctypes.CDLL(LIB_SHIM))
        return _shim
    if _lib is None:
        _lib = _declare(ctypes.CDLL(LIB))
    return _lib


def _declare(L):
    L.ref_geom3d.argtypes = [_I, _I, _I, _I, _P, _I, _I, _I, _F, _F, _P, _F, _F, _P, _P, _P]
    L.ref_geom2d.argtypes = [_I, _I, _I, _P, _I, _I, _F, _P, _F, _F, _P, _P, _P]
    L.ref_cuda_fp3d.argtypes = [_I, _P, _I, _I, _I, _I, _I, _I, _P, _F, _I, _P, _P]
    L.ref_cuda_bp3d.argtypes = [_I, _I, _P, _I, _I, _I, _I, _I, _I, _P, _F, _I, _P, _P]
    L.ref_cuda_cyl.argtypes = [_I, _P, _I, _I, _I, _I, _I, _I, _P, _F, _P, _P]
    L.ref_cuda_sumsqw.argtypes = [_P, _I, _I, _I, _I, _I, _I, _P, _F, _P]
    L.ref_cuda_fdk.argtypes = [_P, _I, _I, _I, _I, _I, _I, _P, _I, _F, _P, _P]
    L.ref_cuda_fp2d.argtypes = [_I, _P, _I, _I, _I, _I, _F, _I, _P, _P]
    L.ref_cuda_bp2d.argtypes = [_I, _P, _I, _I, _I, _I, _F, _I, _I, _P, _P]
    L.ref_gen_filter.argtypes = [_I, _F, _F, _I, _P]
    L.ref_sart2d.argtypes = [_I, _I, _I, _P, _I, _I, _F, _P, _F, _F, _P, _P, _P, _I, _I, _F, _I, _F]
    L.ref_cgm_cone.argtypes = [_I, _I, ctypes.c_size_t, _I, _I, _I, _I, _I, _I, _F, _F, _P, _F, _F, _P, _P]
    return L


def cgm_cone(op, angles, sod, odd, proj, vol, memory=0, gpu_data=True, det_spacing=(1.0, 1.0)):
    """The reference's CompositeGeometryManager doFP (op 'fp': proj = A vol)
    or doBP (op 'bp': vol = B proj) on a circular cone geometry, MODE_SET.
    gpu_data: proj and vol are float32 CUDA tensors linked as the reference's
    GPU data (the direct_FP3D / direct_BP3D path); else float32 numpy arrays in
    the reference's host data objects (create_sino3d_gpu).  memory: the GPU
    memory limit under which the manager splits the job (0: none)."""
    ang = np.ascontiguousarray(angles, dtype=np.float32)
    nv, na, nu = proj.shape
    nz, ny, nx = vol.shape
    if gpu_data:
        import torch
        torch.cuda.synchronize()
        pp, vp = proj.data_ptr(), vol.data_ptr()
    else:
        assert proj.dtype == np.float32 and vol.dtype == np.float32
        assert proj.flags.c_contiguous and vol.flags.c_contiguous
        pp, vp = proj.ctypes.data, vol.ctypes.data
    rc = lib().ref_cgm_cone(0 if op == 'fp' else 1, int(bool(gpu_data)), int(memory), nx, ny, nz, na, nu, nv,
                            det_spacing[0], det_spacing[1], ang.ctypes.data, sod, odd, pp, vp)
    assert rc == 0, "the reference's CompositeGeometryManager failed"


def geom3d(vol_geom, proj_geom):
    """Reference convertAstraGeometry: ((n,12) float64 views, (3,) float32 voxel size)."""
    t = proj_geom['type']
    o = vol_geom['option']
    win = np.array([o['WindowMinX'], o['WindowMaxX'], o['WindowMinY'], o['WindowMaxY'],
                    o['WindowMinZ'], o['WindowMaxZ']], dtype=np.float32)
    rows, cols = proj_geom['DetectorRowCount'], proj_geom['DetectorColCount']
    if 'Vectors' in proj_geom:
        vec = np.ascontiguousarray(proj_geom['Vectors'], dtype=np.float64)
        na = vec.shape[0]
        ang = np.zeros(1, dtype=np.float32)
        sx = sy = sod = odd = 0.0
    else:
        ang = np.ascontiguousarray(proj_geom['ProjectionAngles'], dtype=np.float32).ravel()
        na = ang.size
        vec = np.zeros(12, dtype=np.float64)
        sx, sy = proj_geom['DetectorSpacingX'], proj_geom['DetectorSpacingY']
        sod = proj_geom.get('DistanceOriginSource', 0.0)
        odd = proj_geom.get('DistanceOriginDetector', 0.0)
    views = np.zeros((na, 13 if t == 'cyl_cone_vec' else 12), dtype=np.float64)
    vs = np.zeros(3, dtype=np.float32)
    rc = lib().ref_geom3d(GEOM3D_TYPES[t], vol_geom['GridColCount'], vol_geom['GridRowCount'],
                          vol_geom['GridSliceCount'], win.ctypes.data, na, rows, cols, sx, sy,
                          ang.ctypes.data, sod, odd, vec.ctypes.data, views.ctypes.data, vs.ctypes.data)
    assert rc == 0
    return views, vs


def geom2d(vol_geom, proj_geom):
    """Reference 2D convertAstraGeometry: ((n,6) float32 views, output scale)."""
    t = proj_geom['type']
    o = vol_geom['option']
    win = np.array([o['WindowMinX'], o['WindowMaxX'], o['WindowMinY'], o['WindowMaxY']], dtype=np.float32)
    ndet = proj_geom['DetectorCount']
    if 'Vectors' in proj_geom:
        vec = np.ascontiguousarray(proj_geom['Vectors'], dtype=np.float64)
        na = vec.shape[0]
        ang = np.zeros(1, dtype=np.float32)
        w = sod = odd = 0.0
    else:
        ang = np.ascontiguousarray(proj_geom['ProjectionAngles'], dtype=np.float32).ravel()
        na = ang.size
        vec = np.zeros(6, dtype=np.float64)
        w = proj_geom['DetectorWidth']
        sod = proj_geom.get('DistanceOriginSource', 0.0)
        odd = proj_geom.get('DistanceOriginDetector', 0.0)
    views = np.zeros((na, 6), dtype=np.float32)
    sc = np.zeros(1, dtype=np.float32)
    rc = lib().ref_geom2d(GEOM2D_TYPES[t], vol_geom['GridColCount'], vol_geom['GridRowCount'],
                          win.ctypes.data, na, ndet, w, ang.ctypes.data, sod, odd, vec.ctypes.data,
                          views.ctypes.data, sc.ctypes.data)
    assert rc == 0
    return views, float(sc[0])


# ---------------------------------------------------------------------------
# reference CUDA projectors (need a GPU; device pointers from torch tensors)
# ---------------------------------------------------------------------------

def cuda_fp3d(kind, views, vol, nu, nv, vol_scale=(1.0, 1.0, 1.0), out_scale=1.0, rays=1):
    """Reference ConeFP / Par3DFP on a float32 CUDA tensor vol (z, y, x); returns a new tensor."""
    import torch
    views = np.ascontiguousarray(views, dtype=np.float64)
    vs = np.ascontiguousarray(vol_scale, dtype=np.float32)
    nz, ny, nx = vol.shape
    na = views.shape[0]
    proj = torch.zeros((nv, na, nu), dtype=torch.float32, device=vol.device)
    torch.cuda.synchronize()
    rc = lib().ref_cuda_fp3d(kind, views.ctypes.data, nx, ny, nz, na, nu, nv, vs.ctypes.data, out_scale,
                             rays, vol.data_ptr(), proj.data_ptr())
    assert rc == 0
    torch.cuda.synchronize()
    return proj


def cuda_cyl(op, views, data, vol_shape, nu, nv, vol_scale, out_scale=1.0):
    """Reference cyl_cone_vec projector: op 'fp' (data = volume), 'bp' or
    'bp_matched' (data = projections); returns a new float32 CUDA tensor."""
    import torch
    views = np.ascontiguousarray(views, dtype=np.float64)
    vs = np.ascontiguousarray(vol_scale, dtype=np.float32)
    nz, ny, nx = vol_shape
    na = views.shape[0]
    shape = (nv, na, nu) if op == 'fp' else tuple(vol_shape)
    out = torch.zeros(shape, dtype=torch.float32, device='cuda')
    torch.cuda.synchronize()
    code = {'fp': 0, 'bp': 1, 'bp_matched': 2}[op]
    rc = lib().ref_cuda_cyl(code, views.ctypes.data, nx, ny, nz, na, nu, nv, vs.ctypes.data, out_scale,
                            data.data_ptr(), out.data_ptr())
    assert rc == 0
    torch.cuda.synchronize()
    return out


def cuda_sumsqw(views, vol_shape, nu, nv, vol_scale=(1.0, 1.0, 1.0), out_scale=1.0):
    """Reference Par3DFP_SumSqW ('sum_square_weights'); returns a new float32 CUDA tensor."""
    import torch
    views = np.ascontiguousarray(views, dtype=np.float64)
    vs = np.ascontiguousarray(vol_scale, dtype=np.float32)
    nz, ny, nx = vol_shape
    na = views.shape[0]
    proj = torch.zeros((nv, na, nu), dtype=torch.float32, device='cuda')
    torch.cuda.synchronize()
    rc = lib().ref_cuda_sumsqw(views.ctypes.data, nx, ny, nz, na, nu, nv, vs.ctypes.data, out_scale,
                               proj.data_ptr())
    assert rc == 0
    torch.cuda.synchronize()
    return proj


def cuda_bp3d(kind, views, proj, vol_shape, vol_scale=(1.0, 1.0, 1.0), out_scale=1.0, kernel=0, rays=1):
    import torch
    views = np.ascontiguousarray(views, dtype=np.float64)
    vs = np.ascontiguousarray(vol_scale, dtype=np.float32)
    nv, na, nu = proj.shape
    nz, ny, nx = vol_shape
    vol = torch.zeros(vol_shape, dtype=torch.float32, device=proj.device)
    torch.cuda.synchronize()
    rc = lib().ref_cuda_bp3d(kind, kernel, views.ctypes.data, nx, ny, nz, na, nu, nv, vs.ctypes.data,
                             out_scale, rays, proj.data_ptr(), vol.data_ptr())
    assert rc == 0
    torch.cuda.synchronize()
    return vol


def cuda_fdk(views, proj, vol_shape, vol_scale=(1.0, 1.0, 1.0), short_scan=False, out_scale=1.0):
    """Reference FDK (Ram-Lak); proj is filtered in place (pass a copy)."""
    import torch
    views = np.ascontiguousarray(views, dtype=np.float64)
    vs = np.ascontiguousarray(vol_scale, dtype=np.float32)
    nv, na, nu = proj.shape
    nz, ny, nx = vol_shape
    vol = torch.zeros(vol_shape, dtype=torch.float32, device=proj.device)
    torch.cuda.synchronize()
    rc = lib().ref_cuda_fdk(views.ctypes.data, nx, ny, nz, na, nu, nv, vs.ctypes.data, int(short_scan),
                            out_scale, proj.data_ptr(), vol.data_ptr())
    assert rc == 0
    torch.cuda.synchronize()
    return vol


def cuda_fp2d(kind, views, vol, ndet, out_scale=1.0, rays=1):
    """kind 3 parallel, 4 fan; vol (rows, cols) float32 CUDA tensor."""
    import torch
    views = np.ascontiguousarray(views, dtype=np.float32)
    H, W = vol.shape
    na = views.shape[0]
    sino = torch.zeros((na, ndet), dtype=torch.float32, device=vol.device)
    torch.cuda.synchronize()
    rc = lib().ref_cuda_fp2d(kind, views.ctypes.data, W, H, na, ndet, out_scale, rays, vol.data_ptr(),
                             sino.data_ptr())
    assert rc == 0
    torch.cuda.synchronize()
    return sino


def cuda_bp2d(kind, views, sino, vol_shape, out_scale=1.0, rays=1, fbp=False):
    import torch
    views = np.ascontiguousarray(views, dtype=np.float32)
    na, ndet = sino.shape
    H, W = vol_shape
    vol = torch.zeros(vol_shape, dtype=torch.float32, device=sino.device)
    torch.cuda.synchronize()
    rc = lib().ref_cuda_bp2d(kind, views.ctypes.data, W, H, na, ndet, out_scale, rays, int(fbp),
                             sino.data_ptr(), vol.data_ptr())
    assert rc == 0
    torch.cuda.synchronize()
    return vol


def sart2d(vol_geom, proj_geom, sino, vol0, iterations, min_value=None, max_value=None):
    """Reference SART_CUDA (sequential order, relaxation 1) on host arrays;
    returns the updated volume.  Runs the reference's CUDA code: needs a GPU."""
    t = proj_geom['type']
    o = vol_geom['option']
    win = np.array([o['WindowMinX'], o['WindowMaxX'], o['WindowMinY'], o['WindowMaxY']], dtype=np.float32)
    ndet = proj_geom['DetectorCount']
    if 'Vectors' in proj_geom:
        vec = np.ascontiguousarray(proj_geom['Vectors'], dtype=np.float64)
        na = vec.shape[0]
        ang = np.zeros(1, dtype=np.float32)
        w = sod = odd = 0.0
    else:
        ang = np.ascontiguousarray(proj_geom['ProjectionAngles'], dtype=np.float32).ravel()
        na = ang.size
        vec = np.zeros(6, dtype=np.float64)
        w = proj_geom['DetectorWidth']
        sod = proj_geom.get('DistanceOriginSource', 0.0)
        odd = proj_geom.get('DistanceOriginDetector', 0.0)
    sino = np.ascontiguousarray(sino, dtype=np.float32)
    vol = np.array(vol0, dtype=np.float32, copy=True, order='C')
    rc = lib().ref_sart2d(GEOM2D_TYPES[t], vol_geom['GridColCount'], vol_geom['GridRowCount'], win.ctypes.data, na,
                          ndet, w, ang.ctypes.data, sod, odd, vec.ctypes.data, sino.ctypes.data, vol.ctypes.data,
                          iterations, int(min_value is not None), float(min_value or 0.0),
                          int(max_value is not None), float(max_value or 0.0))
    assert rc == 0
    return vol


class Algo3D:
    """The reference's own 3D algorithm object -- 'SIRT3D_CUDA', 'CGLS3D_CUDA'
    or 'FDK_CUDA' (Ram-Lak) -- for a circular cone geometry over float32 CUDA
    tensors proj (v, angles, u) and vol (z, y, x), linked as the reference's
    GPU data.  run() synchronises the device."""

    TYPES = {'SIRT3D_CUDA': 0, 'CGLS3D_CUDA': 1, 'FDK_CUDA': 2}

    def __init__(self, kind, angles, sod, odd, proj, vol, det_spacing=(1.0, 1.0)):
        L = lib()
        L.ref_algo3d_create.restype = _P
        L.ref_algo3d_create.argtypes = [_I, _I, _I, _I, _I, _I, _I, _F, _F, _P, _F, _F, _P, _P]
        L.ref_algo3d_run.argtypes = [_P, _I]
        L.ref_algo3d_residual.argtypes = [_P, _P]
        L.ref_algo3d_destroy.argtypes = [_P]
        self._L = L
        self._keep = (proj, vol)
        self.angles = np.ascontiguousarray(angles, dtype=np.float32)
        nv, na, nu = proj.shape
        nz, ny, nx = vol.shape
        self.h = L.ref_algo3d_create(self.TYPES[kind], nx, ny, nz, na, nu, nv, det_spacing[0], det_spacing[1],
                                     self.angles.ctypes.data, sod, odd, proj.data_ptr(), vol.data_ptr())
        assert self.h, "the reference refused the algorithm"

    def run(self, iterations=1):
        assert self._L.ref_algo3d_run(self.h, int(iterations)) == 0

    def residual(self):
        v = ctypes.c_float(0.0)
        assert self._L.ref_algo3d_residual(self.h, ctypes.byref(v)) == 0
        return float(v.value)

    def close(self):
        if self.h:
            self._L.ref_algo3d_destroy(self.h)
            self.h = None


# ---------------------------------------------------------------------------
# the reference's CPU 2D path (oracle/_ref/libastra_ref_cpu.so, built without
# CUDA by oracle/ref_cpu.mk; single-threaded, runs without a GPU)
# ---------------------------------------------------------------------------

LIB_CPU = os.path.join(_HERE, "_ref", "libastra_ref_cpu.so")
CPU_KERNELS = {'line': 0, 'linear': 1, 'strip': 2}
_lib_cpu = None


def cpu_available():
    return os.path.exists(LIB_CPU)


def lib_cpu():
    global _lib_cpu
    if _lib_cpu is None:
        L = ctypes.CDLL(LIB_CPU)
        for name in ("refcpu_fp2d", "refcpu_bp2d"):
            getattr(L, name).argtypes = [_I, _I, _I, _I, _I, _I, _F, _P, _F, _F, _P, _P]
        L.refcpu_sirt2d.argtypes = [_I, _I, _I, _I, _I, _I, _F, _P, _F, _F, _P, _P, _I]
        _lib_cpu = L
    return _lib_cpu


def _cpu_args(kind, kernel, shape, angles, ndet, det_width, sod, odd):
    rows, cols = shape
    ang = np.ascontiguousarray(angles, dtype=np.float32)
    geom = {'parallel': 0, 'fanflat': 1}[kind]
    return [geom, CPU_KERNELS[kernel], cols, rows, ang.size, ndet, det_width, ang.ctypes.data, sod, odd], ang


def cpu_fp2d(kind, kernel, vol, angles, ndet, det_width=1.0, sod=0.0, odd=0.0):
    """Reference CPU forward projection ('parallel': line / linear / strip,
    'fanflat': line / strip) of a (rows, cols) float32 volume of unit pixels
    centred on the origin; returns the (angles, ndet) sinogram."""
    vol = np.ascontiguousarray(vol, dtype=np.float32)
    args, ang = _cpu_args(kind, kernel, vol.shape, angles, ndet, det_width, sod, odd)
    sino = np.zeros((ang.size, ndet), dtype=np.float32)
    assert lib_cpu().refcpu_fp2d(*args, vol.ctypes.data, sino.ctypes.data) == 0
    return sino


def cpu_bp2d(kind, kernel, sino, shape, angles, det_width=1.0, sod=0.0, odd=0.0):
    """Reference CPU backprojection of an (angles, ndet) sinogram into a (rows, cols) volume."""
    sino = np.ascontiguousarray(sino, dtype=np.float32)
    args, ang = _cpu_args(kind, kernel, shape, angles, sino.shape[1], det_width, sod, odd)
    vol = np.zeros(shape, dtype=np.float32)
    assert lib_cpu().refcpu_bp2d(*args, sino.ctypes.data, vol.ctypes.data) == 0
    return vol


def cpu_sirt2d(kind, kernel, sino, shape, angles, iterations, det_width=1.0, sod=0.0, odd=0.0, vol0=None):
    """Reference CPU SIRT (CSirtAlgorithm) from vol0 (zeros by default)."""
    sino = np.ascontiguousarray(sino, dtype=np.float32)
    args, ang = _cpu_args(kind, kernel, shape, angles, sino.shape[1], det_width, sod, odd)
    vol = np.zeros(shape, dtype=np.float32) if vol0 is None else np.array(vol0, dtype=np.float32, order='C')
    assert lib_cpu().refcpu_sirt2d(*args, sino.ctypes.data, vol.ctypes.data, int(iterations)) == 0
    return vol


def gen_filter(ref_type, N, d=1.0, parameter=-1.0):
    """The reference's genFilter spectrum (N // 2 + 1 floats) for E_FBPFILTER
    value ref_type (FILTER_ERROR = 0, FILTER_NONE = 1, FILTER_RAMLAK = 2, ...)."""
    out = np.zeros(N // 2 + 1, dtype=np.float32)
    rc = lib().ref_gen_filter(int(ref_type), float(d), float(parameter), int(N), out.ctypes.data)
    if rc != 0:
        raise RuntimeError("genFilter refused filter %d" % ref_type)
    return out
