"""ctypes wrapper of the FP64 oracle (oracle/b2t_oracle.c).

TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and the
CPU-baseline / reference legs of bench.py as the checker.  The product path
(astra-toolbox_b200) never imports this module.

Geometry is taken as the reference's per-view vectors: (n, 12) float64 arrays
for 3D (SConeProjection / SPar3DProjection order), (n, 6) float32 arrays for 2D
(SFanProjection / SParProjection order), already normalised to unit voxels.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(_HERE, "liboracle.so")

PAR3D, CONE = 1, 2
KER_DEFAULT, KER_FDK, KER_2D = 0, 2, 3

_lib = None
_P = ctypes.c_void_p
_L = ctypes.c_long
_I = ctypes.c_int
_D = ctypes.c_double


def build():
    """Compile liboracle.so with the Makefile next to this file."""
    subprocess.check_call(["make", "-s", "-C", _HERE, "liboracle.so"])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = ctypes.CDLL(LIB)
        L.orc_fp3d.argtypes = [_I, _P, _L, _L, _L, _L, _L, _L, _P, _D, _I, _I, _P, _P, _L, _L, _I]
        L.orc_fp3d_transpose.argtypes = [_I, _P, _L, _L, _L, _L, _L, _L, _P, _D, _P, _P]
        L.orc_bp3d.argtypes = [_I, _I, _P, _L, _L, _L, _L, _L, _L, _P, _D, _I, _I, _P, _P, _L, _L, _I]
        L.orc_dominant_axis3d.argtypes = [_I, _P, _L, _L]
        L.orc_fdk_params.argtypes = [_P, _L, _L, _L, _P, _P]
        L.orc_fdk_preweight.argtypes = [_P, _L, _L, _L, _D, _D, _D, _D, _D]
        L.orc_parker_setup.argtypes = [_P, _L, _L, _D, _D, _D, _P, _P, _P]
        L.orc_parker_weight.argtypes = [_P, _L, _L, _L, _D, _D, _D, _P, _D, _D]
        L.orc_ramp_filter_rows.argtypes = [_P, _L, _L, _I]
        L.orc_ramp_taps.argtypes = [_L, _P]
        L.orc_par_fp.argtypes = [_P, _L, _L, _L, _L, _D, _I, _I, _P, _P]
        L.orc_par_bp.argtypes = [_P, _L, _L, _L, _L, _D, _I, _I, _P, _P]
        L.orc_fan_fp.argtypes = [_P, _L, _L, _L, _L, _D, _I, _I, _P, _P]
        L.orc_fan_bp.argtypes = [_P, _L, _L, _L, _L, _D, _I, _I, _I, _P, _P]
        _lib = L
    return _lib


def _c(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


def nthreads_default():
    return os.cpu_count() or 1


def fp3d(kind, views, vol, det_u, det_v, vol_scale=(1.0, 1.0, 1.0), out_scale=1.0, rays=1,
         tex8=False, angles=None, nthreads=None):
    """Forward projection; returns float64 [det_v][n_angles][det_u].

    angles: optional (begin, end) range of views to compute (others left 0)."""
    views = _c(views, np.float64)
    vol = _c(vol, np.float32)
    nz, ny, nx = vol.shape
    na = views.shape[0]
    proj = np.zeros((det_v, na, det_u), dtype=np.float64)
    vs = _c(vol_scale, np.float64)
    a0, a1 = (0, na) if angles is None else angles
    rc = lib().orc_fp3d(kind, views.ctypes.data, nx, ny, nz, na, det_u, det_v, vs.ctypes.data,
                        out_scale, rays, int(tex8), vol.ctypes.data, proj.ctypes.data, a0, a1,
                        nthreads or nthreads_default())
    assert rc == 0
    return proj


def fp3d_transpose(kind, views, proj, vol_shape, vol_scale=(1.0, 1.0, 1.0), out_scale=1.0):
    """Exact transpose of fp3d (single thread); returns float64 [z][y][x]."""
    views = _c(views, np.float64)
    proj = _c(proj, np.float64)
    nv, na, nu = proj.shape
    nz, ny, nx = vol_shape
    vol = np.zeros(vol_shape, dtype=np.float64)
    vs = _c(vol_scale, np.float64)
    rc = lib().orc_fp3d_transpose(kind, views.ctypes.data, nx, ny, nz, na, nu, nv, vs.ctypes.data,
                                  out_scale, proj.ctypes.data, vol.ctypes.data)
    assert rc == 0
    return vol


def bp3d(kind, views, proj, vol_shape, vol_scale=(1.0, 1.0, 1.0), out_scale=1.0, kernel=KER_DEFAULT,
         rays=1, tex8=False, z_range=None, nthreads=None):
    """Backprojection; returns float64 [z][y][x] (slices outside z_range left 0)."""
    views = _c(views, np.float64)
    proj = _c(proj, np.float32)
    nv, na, nu = proj.shape
    nz, ny, nx = vol_shape
    vol = np.zeros(vol_shape, dtype=np.float64)
    vs = _c(vol_scale, np.float64)
    z0, z1 = (0, nz) if z_range is None else z_range
    rc = lib().orc_bp3d(kind, kernel, views.ctypes.data, nx, ny, nz, na, nu, nv, vs.ctypes.data,
                        out_scale, rays, int(tex8), proj.ctypes.data, vol.ctypes.data, z0, z1,
                        nthreads or nthreads_default())
    assert rc == 0
    return vol


def dominant_axis3d(kind, view, det_u, det_v):
    v = _c(view, np.float64)
    return lib().orc_dominant_axis3d(kind, v.ctypes.data, det_u, det_v)


def fdk_params(views, det_u, det_v):
    """(src_origin, det_origin, det_usize, det_vsize, zshift), angles (float32)."""
    views = _c(views, np.float64)
    na = views.shape[0]
    out = np.zeros(5, dtype=np.float32)
    ang = np.zeros(na, dtype=np.float32)
    lib().orc_fdk_params(views.ctypes.data, na, det_u, det_v, out.ctypes.data, ang.ctypes.data)
    return out, ang


def fdk_weight(proj, views, short_scan=False):
    """FDK pre-weighting (and Parker weighting if short_scan) of float64 proj in place."""
    nv, na, nu = proj.shape
    p, ang = fdk_params(views, nu, nv)
    assert proj.dtype == np.float64 and proj.flags.c_contiguous
    lib().orc_fdk_preweight(proj.ctypes.data, na, nu, nv, float(p[0]), float(p[1]), float(p[4]),
                            float(p[2]), float(p[3]))
    if short_scan and na > 1:
        rel = np.zeros(na, dtype=np.float32)
        sc = np.zeros(1, dtype=np.float32)
        cf = np.zeros(1, dtype=np.float32)
        lib().orc_parker_setup(ang.ctypes.data, na, nu, float(p[0]), float(p[1]), float(p[2]),
                               rel.ctypes.data, sc.ctypes.data, cf.ctypes.data)
        lib().orc_parker_weight(proj.ctypes.data, na, nu, nv, float(p[0]), float(p[1]), float(p[2]),
                                rel.ctypes.data, float(sc[0]), float(cf[0]))
    return proj


def ramp_taps(n):
    t = np.zeros(n, dtype=np.float64)
    lib().orc_ramp_taps(n, t.ctypes.data)
    return t


def ramp_filter_rows(rows, nthreads=None):
    """Ram-Lak filter of every row of a float64 array (last axis), in place."""
    assert rows.dtype == np.float64 and rows.flags.c_contiguous
    n = rows.shape[-1]
    lib().orc_ramp_filter_rows(rows.ctypes.data, rows.size // n, n, nthreads or nthreads_default())
    return rows


def fdk(views, proj, vol_shape, vol_scale=(1.0, 1.0, 1.0), short_scan=False, out_scale=1.0,
        nthreads=None):
    """FDK: weight, ramp-filter along u, cone BP with FDK weighting (float64)."""
    p = np.array(proj, dtype=np.float64, copy=True)
    fdk_weight(p, views, short_scan)
    ramp_filter_rows(p, nthreads)
    return bp3d(CONE, views, p.astype(np.float32), vol_shape, vol_scale, out_scale, kernel=KER_FDK,
                nthreads=nthreads)


def par_fp(views, vol, ndet, out_scale=1.0, rays=1, tex8=False):
    views = _c(views, np.float32)
    vol = _c(vol, np.float32)
    H, W = vol.shape
    na = views.shape[0]
    sino = np.zeros((na, ndet), dtype=np.float64)
    lib().orc_par_fp(views.ctypes.data, na, ndet, W, H, out_scale, rays, int(tex8), vol.ctypes.data,
                     sino.ctypes.data)
    return sino


def par_bp(views, sino, vol_shape, out_scale=1.0, rays=1, tex8=False):
    views = _c(views, np.float32)
    sino = _c(sino, np.float32)
    na, ndet = sino.shape
    H, W = vol_shape
    vol = np.zeros(vol_shape, dtype=np.float64)
    lib().orc_par_bp(views.ctypes.data, na, ndet, W, H, out_scale, rays, int(tex8), sino.ctypes.data,
                     vol.ctypes.data)
    return vol


def fan_fp(views, vol, ndet, out_scale=1.0, rays=1, tex8=False):
    views = _c(views, np.float32)
    vol = _c(vol, np.float32)
    H, W = vol.shape
    na = views.shape[0]
    sino = np.zeros((na, ndet), dtype=np.float64)
    lib().orc_fan_fp(views.ctypes.data, na, ndet, W, H, out_scale, rays, int(tex8), vol.ctypes.data,
                     sino.ctypes.data)
    return sino


def fan_bp(views, sino, vol_shape, out_scale=1.0, rays=1, fbp=False, tex8=False):
    views = _c(views, np.float32)
    sino = _c(sino, np.float32)
    na, ndet = sino.shape
    H, W = vol_shape
    vol = np.zeros(vol_shape, dtype=np.float64)
    lib().orc_fan_bp(views.ctypes.data, na, ndet, W, H, out_scale, rays, int(fbp), int(tex8),
                     sino.ctypes.data, vol.ctypes.data)
    return vol
