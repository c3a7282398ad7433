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
        L.orc_par3d_sumsqw.argtypes = [_P, _L, _L, _L, _L, _L, _L, _P, _D, _P]
        L.orc_bp3d.argtypes = [_I, _I, _P, _L, _L, _L, _L, _L, _L, _P, _D, _I, _I, _P, _P, _L, _L, _I]
        L.orc_dominant_axis3d.argtypes = [_I, _P, _L, _L]
        L.orc_fdk_params.argtypes = [_P, _L, _L, _L, _P, _P]
        L.orc_fdk_preweight.argtypes = [_P, _L, _L, _L, _D, _D, _D, _D, _D]
        L.orc_parker_setup.argtypes = [_P, _L, _L, _D, _D, _D, _P, _P, _P]
        L.orc_parker_weight.argtypes = [_P, _L, _L, _L, _D, _D, _D, _P, _D, _D]
        L.orc_ramp_filter_rows.argtypes = [_P, _L, _L, _I]
        L.orc_ramp_taps.argtypes = [_L, _P]
        L.orc_toeplitz_rows.argtypes = [_P, _L, _L, _P, _L, _L, _I]
        L.orc_par_fp.argtypes = [_P, _L, _L, _L, _L, _D, _I, _I, _P, _P]
        L.orc_par_bp.argtypes = [_P, _L, _L, _L, _L, _D, _I, _I, _P, _P]
        L.orc_fan_fp.argtypes = [_P, _L, _L, _L, _L, _D, _I, _I, _P, _P]
        L.orc_fan_bp.argtypes = [_P, _L, _L, _L, _L, _D, _I, _I, _I, _P, _P]
        L.orc_cylcone_fp.argtypes = [_P, _L, _L, _L, _L, _L, _L, _P, _D, _I, _P, _P]
        L.orc_cylcone_fp_transpose.argtypes = [_P, _L, _L, _L, _L, _L, _L, _P, _D, _P, _P]
        L.orc_cylcone_bp.argtypes = [_P, _L, _L, _L, _L, _L, _L, _P, _D, _I, _P, _P]
        L.orc_sart2d.argtypes = [_I, _P, _L, _L, _L, _L, _D, _I, _P, _L, _L, _L, _D, _I, _D, _I, _D, _I, _P, _P, _P]
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


def par3d_sumsqw(views, vol_shape, det_u, det_v, vol_scale=(1.0, 1.0, 1.0), out_scale=1.0):
    """'sum_square_weights' forward projection of a parallel-beam geometry
    (Par3DFP_SumSqW); returns float64 [det_v][n_angles][det_u]."""
    views = _c(views, np.float64)
    nz, ny, nx = vol_shape
    na = views.shape[0]
    proj = np.zeros((det_v, na, det_u), dtype=np.float64)
    vs = _c(vol_scale, np.float64)
    rc = lib().orc_par3d_sumsqw(views.ctypes.data, nx, ny, nz, na, det_u, det_v, vs.ctypes.data, out_scale,
                                proj.ctypes.data)
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


# E_FBPFILTER order (include/astra/Filters.h:43-66) without FILTER_ERROR
FILTERS = ['none', 'ram-lak', 'shepp-logan', 'cosine', 'hamming', 'hann', 'tukey', 'lanczos', 'triangular',
           'gaussian', 'barlett-hann', 'blackman', 'nuttall', 'blackman-harris', 'blackman-nuttall', 'flat-top',
           'kaiser', 'parzen', 'projection', 'sinogram', 'rprojection', 'rsinogram']


def _next_pow2(n):
    x = 1
    while x < n:
        x *= 2
    return x


def filter_spectrum(name, N, d=1.0, parameter=-1.0):
    """genFilter (src/Filters.cpp:131-488) in FP64 on bins 0 .. N/2: twice the
    real DFT of the Ram-Lak spatial taps (generateRampFilter, Filters.cpp:
    41-69), times the window of the named type on bins >= 1, zero where
    w = 2 pi f / N exceeds pi d."""
    F = N // 2 + 1
    i = np.arange(N)
    h = np.zeros(N)
    odd = (i % 2) == 1
    j = np.where(2 * i > N, N - i, i)
    h[odd] = -1.0 / (np.pi * j[odd]) ** 2
    h[0] = 0.25
    f = np.arange(F)
    R = 2.0 * (np.cos(2 * np.pi * np.outer(f, i) / N) @ h)
    n = f[1:].astype(np.float64)
    w = 2 * np.pi * f / N
    nm1 = F - 1.0
    if name == 'ram-lak':
        win = np.ones(F - 1)
    elif name == 'shepp-logan':
        x = w[1:] / 2 / d
        win = np.sin(x) / x
    elif name == 'cosine':
        win = np.cos(w[1:] / 2 / d)
    elif name == 'hamming':
        win = 0.54 + 0.46 * np.cos(w[1:] / d)
    elif name == 'hann':
        win = (1 + np.cos(w[1:] / d)) / 2
    elif name == 'tukey':
        alpha = 0.5 if parameter < 0 else parameter
        half = F / 2.0
        a, den = alpha * half, (1 - alpha) * half
        inside = (half - a <= n) & (n <= half + a)
        win = np.where(inside, 1.0, 0.5 * (1 + np.cos(np.pi * (n - a) / den)))
    elif name == 'lanczos':
        x = np.pi * (2 * n / nm1 - 1)
        win = np.where(np.abs(x) > 0.001, np.sin(x) / np.where(x == 0, 1, x), 1.0)
    elif name == 'triangular':
        win = 2 / nm1 * (nm1 / 2 - np.abs(n - nm1 / 2))
    elif name == 'gaussian':
        sigma = 0.4 if parameter < 0 else parameter
        q = (F - 1) / 2.0
        win = np.exp(-0.5 * ((n - q) / (sigma * q)) ** 2)
    elif name == 'barlett-hann':
        win = 0.62 - 0.48 * np.abs(n / nm1 - 0.5) - 0.38 * np.cos(2 * np.pi * n / nm1)
    elif name == 'blackman':
        alpha = 0.16 if parameter < 0 else parameter
        win = (1 - alpha) / 2 - 0.5 * np.cos(np.pi * n / nm1) + alpha / 2 * np.cos(2 * np.pi * n / nm1)
    elif name in ('nuttall', 'blackman-harris', 'blackman-nuttall', 'flat-top'):
        a = {'nuttall': (0.355768, 0.487396, 0.144232, 0.012604, 0.0),
             'blackman-harris': (0.35875, 0.48829, 0.14128, 0.01168, 0.0),
             'blackman-nuttall': (0.3635819, 0.4891775, 0.1365995, 0.0106411, 0.0),
             'flat-top': (1.0, 1.93, 1.29, 0.388, 0.032)}[name]
        x = np.pi * n / nm1
        win = a[0] - a[1] * np.cos(2 * x) + a[2] * np.cos(4 * x) - a[3] * np.cos(6 * x) + a[4] * np.cos(8 * x)
    elif name == 'kaiser':
        from scipy.special import j0
        alpha = 3.0 if parameter < 0 else parameter
        s = 2 * n / nm1 - 1
        win = j0(np.pi * alpha * np.sqrt(np.clip(1 - s * s, 0, None))) / j0(np.pi * alpha)
    elif name == 'parzen':
        q = n / nm1
        win = np.where(q <= 0.5, 1 - 6 * q * q * (1 - q), 2 * (1 - q) ** 3)
    else:
        raise ValueError("no spectrum for filter %r" % name)
    G = R.copy()
    G[1:] *= win
    G[w > np.pi * d] = 0.0
    return G


def _spectrum_taps(G, N, n):
    f = np.arange(1, N // 2)
    dd = np.arange(n)
    g = (G[0] + G[N // 2] * np.where(dd % 2 == 1, -1.0, 1.0)
         + 2 * (np.cos(2 * np.pi * np.outer(dd, f) / N) @ G[1:N // 2])) / N
    return np.concatenate([g[:0:-1], g])


def filter_taps(name, n, n_views=1, d=1.0, parameter=-1.0, custom=None):
    """Exact Toeplitz taps (sets, 2n-1) of a filter for rows of n samples, the
    reference's zero-padded FFT filtering (cuda/2d/fft.cu:338-595): spectral
    types from filter_spectrum, 'projection' / 'sinogram' from the custom
    spectrum rows, 'rprojection' / 'rsinogram' from the custom spatial rows
    centred on element width // 2."""
    N = _next_pow2(2 * n)
    if name in ('projection', 'sinogram'):
        c = np.atleast_2d(np.asarray(custom, dtype=np.float64))
        return np.array([_spectrum_taps(row, N, n) for row in c])
    if name in ('rprojection', 'rsinogram'):
        c = np.atleast_2d(np.asarray(custom, dtype=np.float64))
        W = c.shape[1]
        used = min(W, N)
        start = (W - used) // 2
        out = []
        for row in c:
            s = np.zeros(N)
            for i in range(start, start + used):
                s[(i + N - W // 2) % N] = row[i]
            out.append(s[np.arange(-(n - 1), n) % N])
        return np.array(out)
    return _spectrum_taps(filter_spectrum(name, N, d, parameter), N, n)[None, :]


def toeplitz_filter_rows(rows, taps, set_mod=1, nthreads=None):
    """Filter every row of a float64 array in place with taps (sets, 2n-1);
    with several sets, row r uses set r % set_mod."""
    assert rows.dtype == np.float64 and rows.flags.c_contiguous
    n = rows.shape[-1]
    t = _c(taps, np.float64)
    assert t.shape[-1] == 2 * n - 1
    nsets = t.shape[0] if t.ndim == 2 else 1
    lib().orc_toeplitz_rows(rows.ctypes.data, rows.size // n, n, t.ctypes.data, nsets, set_mod,
                            nthreads or nthreads_default())
    return rows


def fdk(views, proj, vol_shape, vol_scale=(1.0, 1.0, 1.0), short_scan=False, out_scale=1.0,
        nthreads=None, taps=None):
    """FDK: weight, filter along u (Ram-Lak, or the given taps), cone BP with
    FDK weighting (float64)."""
    p = np.array(proj, dtype=np.float64, copy=True)
    fdk_weight(p, views, short_scan)
    if taps is None:
        ramp_filter_rows(p, nthreads)
    else:
        toeplitz_filter_rows(p, taps, set_mod=p.shape[1], nthreads=nthreads)
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


def sart2d(kind, views, sino, vol0, out_scale, iterations, order=None, iter0=0, lam=1.0, min_value=None,
           max_value=None, mask=None, rays=1, tex8=False):
    """SART_CUDA's single-view steps (kind 3 parallel, 4 fan) from vol0;
    returns the float32 volume (the state is float, as in the reference)."""
    views = _c(views, np.float32)
    sino = _c(sino, np.float32)
    na, ndet = sino.shape
    vol = np.array(vol0, dtype=np.float32, copy=True, order='C')
    H, W = vol.shape
    o = None if order is None else _c(order, np.int32)
    m = None if mask is None else _c(mask, np.float32)
    rc = lib().orc_sart2d(kind, views.ctypes.data, na, ndet, W, H, out_scale, rays,
                          None if o is None else o.ctypes.data, 0 if o is None else o.size, iter0, iterations,
                          lam, int(min_value is not None), float(min_value or 0.0), int(max_value is not None),
                          float(max_value or 0.0), int(tex8), sino.ctypes.data,
                          None if m is None else m.ctypes.data, vol.ctypes.data)
    assert rc == 0
    return vol


def cylcone_fp(views, vol, det_u, det_v, vol_scale, out_scale=1.0, tex8=False):
    """cyl_cone_vec forward projection (ConeCylFP); views (n, 13) in world
    units centred on the volume; returns float64 [det_v][n][det_u]."""
    views = _c(views, np.float64)
    vol = _c(vol, np.float32)
    nz, ny, nx = vol.shape
    na = views.shape[0]
    proj = np.zeros((det_v, na, det_u), dtype=np.float64)
    vs = _c(vol_scale, np.float64)
    rc = lib().orc_cylcone_fp(views.ctypes.data, nx, ny, nz, na, det_u, det_v, vs.ctypes.data, out_scale,
                              int(tex8), vol.ctypes.data, proj.ctypes.data)
    assert rc == 0
    return proj


def cylcone_fp_transpose(views, proj, vol_shape, vol_scale, out_scale=1.0):
    """Exact transpose of cylcone_fp; returns float64 [z][y][x]."""
    views = _c(views, np.float64)
    proj = _c(proj, np.float64)
    nv, na, nu = proj.shape
    nz, ny, nx = vol_shape
    vol = np.zeros(vol_shape, dtype=np.float64)
    vs = _c(vol_scale, np.float64)
    rc = lib().orc_cylcone_fp_transpose(views.ctypes.data, nx, ny, nz, na, nu, nv, vs.ctypes.data, out_scale,
                                        proj.ctypes.data, vol.ctypes.data)
    assert rc == 0
    return vol


def cylcone_bp(views, proj, vol_shape, vol_scale, out_scale=1.0, tex8=False):
    """cyl_cone_vec voxel-driven backprojection (ConeCylBP); float64 [z][y][x]."""
    views = _c(views, np.float64)
    proj = _c(proj, np.float32)
    nv, na, nu = proj.shape
    nz, ny, nx = vol_shape
    vol = np.zeros(vol_shape, dtype=np.float64)
    vs = _c(vol_scale, np.float64)
    rc = lib().orc_cylcone_bp(views.ctypes.data, nx, ny, nz, na, nu, nv, vs.ctypes.data, out_scale, int(tex8),
                              proj.ctypes.data, vol.ctypes.data)
    assert rc == 0
    return vol


def bp3d_slices(kind, views, proj, vol_shape, slices, vol_scale=(1.0, 1.0, 1.0), out_scale=1.0,
                kernel=KER_DEFAULT, nthreads=None):
    """Backprojection of single z-slices of a (nz, ny, nx) volume; returns
    float64 [len(slices)][y][x].  Each slice is backprojected as a one-slice
    volume centred on the origin, with the views moved along z by the slice
    centre's offset from the volume centre (the source point of a cone view
    and the detector origin; a parallel view's ray direction stays), so a
    full-size check holds one slice instead of the whole volume in memory."""
    views = _c(views, np.float64)
    nz, ny, nx = vol_shape
    out = np.zeros((len(slices), ny, nx), dtype=np.float64)
    for i, z in enumerate(slices):
        zc = float(z) + 0.5 - 0.5 * nz
        w = views.copy()
        if kind == CONE:
            w[:, 2] -= zc
        w[:, 5] -= zc
        out[i] = bp3d(kind, w, proj, (1, ny, nx), vol_scale, out_scale, kernel, nthreads=nthreads)[0]
    return out


def cone_views(angles, det_cols, det_rows, src_origin, origin_det, det_spacing_x=1.0, det_spacing_y=1.0):
    """Per-view vectors of a circular cone geometry for a volume of unit voxels
    centred on the origin (genConeProjections, src/GeometryUtil3D.cpp:42-83;
    convertAstraGeometry is then the identity): (n, 12) float64, the float32
    angles promoted to double as the reference does.  numpy's cos / sin may
    differ from the C library's in the last bit, so this is for workloads
    that need the geometry without the reference build, not for bit-exact
    checks."""
    a = np.asarray(angles, dtype=np.float32).astype(np.float64)
    c, s = np.cos(a), np.sin(a)
    sod, odd = float(src_origin), float(origin_det)
    du, dv = float(det_spacing_x), float(det_spacing_y)
    out = np.zeros((a.size, 12), dtype=np.float64)

    def rot(k, bx, by, bz):
        out[:, k] = bx * c - by * s
        out[:, k + 1] = bx * s + by * c
        out[:, k + 2] = bz

    rot(0, 0.0, -sod, 0.0)
    rot(3, det_cols * du * -0.5, odd, det_rows * dv * -0.5)
    rot(6, du, 0.0, 0.0)
    rot(9, 0.0, 0.0, dv)
    return out
