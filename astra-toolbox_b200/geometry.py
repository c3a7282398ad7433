"""ASTRA geometry dictionaries -> normalised per-view vectors for libb2tomo.

The dictionaries are the ones astra.create_vol_geom / astra.create_proj_geom
produce (python/astra/creators.py:52-330).  Scalars are rounded to float32 the
way the reference's geometry objects store them (ProjectionGeometry3D.h:77-86,
VolumeGeometry3D.h:81-110), then the library builds and normalises the views
with the reference's own arithmetic (src/GeometryUtil3D.cpp, GeometryUtil2D.cpp).
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import AstraError


def _f32(x):
    return float(np.float32(x))


# ---------------------------------------------------------------------------
# creators (python/astra/creators.py:52-330)
# ---------------------------------------------------------------------------

def create_vol_geom(*varargin):
    """Same call forms and dictionary as astra.create_vol_geom."""
    vol_geom = {'option': {}}
    n = len(varargin)
    if n == 1 and isinstance(varargin[0], int):
        vol_geom['GridRowCount'] = varargin[0]
        vol_geom['GridColCount'] = varargin[0]
    elif n == 1 and len(varargin[0]) == 2:
        vol_geom['GridRowCount'] = varargin[0][0]
        vol_geom['GridColCount'] = varargin[0][1]
    elif n == 1 and len(varargin[0]) == 3:
        vol_geom['GridRowCount'] = varargin[0][0]
        vol_geom['GridColCount'] = varargin[0][1]
        vol_geom['GridSliceCount'] = varargin[0][2]
    elif n == 2:
        vol_geom['GridRowCount'] = varargin[0]
        vol_geom['GridColCount'] = varargin[1]
    elif n == 3:
        vol_geom['GridRowCount'] = varargin[0]
        vol_geom['GridColCount'] = varargin[1]
        vol_geom['GridSliceCount'] = varargin[2]
    elif n == 6:
        vol_geom['GridRowCount'] = varargin[0]
        vol_geom['GridColCount'] = varargin[1]
        o = vol_geom['option']
        o['WindowMinX'], o['WindowMaxX'], o['WindowMinY'], o['WindowMaxY'] = varargin[2:6]
    elif n == 9:
        vol_geom['GridRowCount'] = varargin[0]
        vol_geom['GridColCount'] = varargin[1]
        vol_geom['GridSliceCount'] = varargin[2]
        o = vol_geom['option']
        (o['WindowMinX'], o['WindowMaxX'], o['WindowMinY'], o['WindowMaxY'],
         o['WindowMinZ'], o['WindowMaxZ']) = varargin[3:9]
    else:
        raise AstraError(1, "create_vol_geom: unsupported argument list")
    o = vol_geom['option']
    if 'WindowMinX' not in o:
        o['WindowMinX'] = -vol_geom['GridColCount'] / 2.
        o['WindowMaxX'] = vol_geom['GridColCount'] / 2.
        o['WindowMinY'] = -vol_geom['GridRowCount'] / 2.
        o['WindowMaxY'] = vol_geom['GridRowCount'] / 2.
        if 'GridSliceCount' in vol_geom:
            o['WindowMinZ'] = -vol_geom['GridSliceCount'] / 2.
            o['WindowMaxZ'] = vol_geom['GridSliceCount'] / 2.
    return vol_geom


def create_proj_geom(intype, *args):
    """Same call forms and dictionary as astra.create_proj_geom (flat-panel
    types and cyl_cone_vec)."""
    need = {'parallel': 3, 'parallel_vec': 2, 'fanflat': 5, 'fanflat_vec': 2,
            'parallel3d': 5, 'cone': 7, 'cone_vec': 3, 'parallel3d_vec': 3, 'cyl_cone_vec': 3}
    if intype not in need:
        raise AstraError(2, "create_proj_geom: unsupported geometry type %r" % (intype,))
    if len(args) < need[intype]:
        raise AstraError(1, "Not enough variables for create_proj_geom(%s, ...)" % intype)
    if intype == 'parallel':
        return {'type': 'parallel', 'DetectorWidth': args[0], 'DetectorCount': args[1],
                'ProjectionAngles': args[2]}
    if intype in ('parallel_vec', 'fanflat_vec'):
        if args[1].shape[1] != 6:
            raise AstraError(1, 'V should be a Nx6 matrix, with N the number of projections')
        return {'type': intype, 'DetectorCount': args[0], 'Vectors': args[1]}
    if intype == 'fanflat':
        return {'type': 'fanflat', 'DetectorWidth': args[0], 'DetectorCount': args[1],
                'ProjectionAngles': args[2], 'DistanceOriginSource': args[3],
                'DistanceOriginDetector': args[4]}
    if intype == 'parallel3d':
        return {'type': 'parallel3d', 'DetectorSpacingX': args[0], 'DetectorSpacingY': args[1],
                'DetectorRowCount': args[2], 'DetectorColCount': args[3], 'ProjectionAngles': args[4]}
    if intype == 'cone':
        return {'type': 'cone', 'DetectorSpacingX': args[0], 'DetectorSpacingY': args[1],
                'DetectorRowCount': args[2], 'DetectorColCount': args[3], 'ProjectionAngles': args[4],
                'DistanceOriginSource': args[5], 'DistanceOriginDetector': args[6]}
    # cone_vec, parallel3d_vec (12 columns), cyl_cone_vec (13: the radius last)
    ncol = 13 if intype == 'cyl_cone_vec' else 12
    if np.asarray(args[2]).ndim != 2 or np.asarray(args[2]).shape[1] != ncol:
        raise AstraError(1, 'V should be a Nx%d matrix, with N the number of projections' % ncol)
    return {'type': intype, 'DetectorRowCount': args[0], 'DetectorColCount': args[1], 'Vectors': args[2]}


# ---------------------------------------------------------------------------
# shapes
# ---------------------------------------------------------------------------

def is_3d_vol(vol_geom):
    return 'GridSliceCount' in vol_geom


def vol_shape(vol_geom):
    """numpy shape of a volume: (slices, rows, cols) in 3D, (rows, cols) in 2D."""
    if is_3d_vol(vol_geom):
        return (vol_geom['GridSliceCount'], vol_geom['GridRowCount'], vol_geom['GridColCount'])
    return (vol_geom['GridRowCount'], vol_geom['GridColCount'])


def n_angles(proj_geom):
    if 'Vectors' in proj_geom:
        return int(np.asarray(proj_geom['Vectors']).shape[0])
    return int(np.asarray(proj_geom['ProjectionAngles']).size)


def proj_shape(proj_geom):
    """numpy shape of projection data: (rows, angles, cols) in 3D, (angles, dets) in 2D."""
    t = proj_geom['type']
    if t in ('parallel3d', 'cone', 'cone_vec', 'parallel3d_vec', 'cyl_cone_vec'):
        return (proj_geom['DetectorRowCount'], n_angles(proj_geom), proj_geom['DetectorColCount'])
    return (n_angles(proj_geom), proj_geom['DetectorCount'])


# ---------------------------------------------------------------------------
# conversion to the C ABI
# ---------------------------------------------------------------------------

class Geometry3D:
    """A normalised b2t_geom3d plus the view array it points to."""

    def __init__(self, vol_geom, proj_geom):
        lib = _lib.load()
        t = proj_geom['type']
        if t not in ('parallel3d', 'cone', 'cone_vec', 'parallel3d_vec', 'cyl_cone_vec'):
            raise AstraError(2, "3D projector needs a 3D projection geometry, got %r" % t)
        if not is_3d_vol(vol_geom):
            raise AstraError(1, "3D projector needs a 3D volume geometry")
        if t == 'cyl_cone_vec':
            self._init_cyl(vol_geom, proj_geom)
            return
        self.kind = _lib.GEOM_CONE if t in ('cone', 'cone_vec') else _lib.GEOM_PAR3D
        rows, na, cols = proj_shape(proj_geom)
        views = (_lib.View3D * na)()
        if t in ('cone', 'parallel3d'):
            ang = np.ascontiguousarray(np.asarray(proj_geom['ProjectionAngles'], dtype=np.float32).ravel())
            if t == 'cone':
                _lib.check(lib.b2t_cone_views(na, cols, rows, _f32(proj_geom['DistanceOriginSource']),
                                              _f32(proj_geom['DistanceOriginDetector']),
                                              _f32(proj_geom['DetectorSpacingX']),
                                              _f32(proj_geom['DetectorSpacingY']), _lib.ptr(ang), views))
            else:
                _lib.check(lib.b2t_par3d_views(na, cols, rows, _f32(proj_geom['DetectorSpacingX']),
                                               _f32(proj_geom['DetectorSpacingY']), _lib.ptr(ang), views))
        else:
            vec = np.ascontiguousarray(np.asarray(proj_geom['Vectors'], dtype=np.float64))
            _lib.check(lib.b2t_vec_views3d(na, cols, rows, _lib.ptr(vec), views))
        o = vol_geom['option']
        vg = _lib.VolGeom3D(vol_geom['GridColCount'], vol_geom['GridRowCount'], vol_geom['GridSliceCount'],
                            _f32(o['WindowMinX']), _f32(o['WindowMaxX']), _f32(o['WindowMinY']),
                            _f32(o['WindowMaxY']), _f32(o['WindowMinZ']), _f32(o['WindowMaxZ']))
        vs = (ctypes.c_float * 3)()
        _lib.check(lib.b2t_normalize_views3d(ctypes.byref(vg), self.kind, na, views, vs))
        self.views = views
        self.vol_scale = tuple(vs)
        self.dims = _lib.Dims3D(vol_geom['GridColCount'], vol_geom['GridRowCount'], vol_geom['GridSliceCount'],
                                na, cols, rows)
        self.c = _lib.Geom3D(self.kind, self.dims, (ctypes.c_float * 3)(*vs), views)
        self.vol_shape = vol_shape(vol_geom)
        self.proj_shape = (rows, na, cols)

    def _init_cyl(self, vol_geom, proj_geom):
        """cyl_cone_vec: views translated to the volume centre, not scaled
        (b2t_normalize_views3d_cyl); self.c is a b2t_geom3d_cyl."""
        lib = _lib.load()
        self.kind = _lib.GEOM_CYLCONE
        rows, na, cols = proj_shape(proj_geom)
        vec = np.ascontiguousarray(np.asarray(proj_geom['Vectors'], dtype=np.float64))
        if vec.ndim != 2 or vec.shape != (na, 13):
            raise AstraError(1, "cyl_cone_vec Vectors must be an (n, 13) array")
        views = (_lib.View3DCyl * na)()
        ctypes.memmove(views, vec.ctypes.data, vec.nbytes)
        o = vol_geom['option']
        vg = _lib.VolGeom3D(vol_geom['GridColCount'], vol_geom['GridRowCount'], vol_geom['GridSliceCount'],
                            _f32(o['WindowMinX']), _f32(o['WindowMaxX']), _f32(o['WindowMinY']),
                            _f32(o['WindowMaxY']), _f32(o['WindowMinZ']), _f32(o['WindowMaxZ']))
        vs = (ctypes.c_float * 3)()
        _lib.check(lib.b2t_normalize_views3d_cyl(ctypes.byref(vg), na, views, vs))
        self.views = views
        self.vol_scale = tuple(vs)
        self.dims = _lib.Dims3D(vol_geom['GridColCount'], vol_geom['GridRowCount'], vol_geom['GridSliceCount'],
                                na, cols, rows)
        self.c = _lib.Geom3DCyl(self.dims, (ctypes.c_float * 3)(*vs), views)
        self.vol_shape = vol_shape(vol_geom)
        self.proj_shape = (rows, na, cols)

    def views_array(self):
        """Per-view vectors as an (n, 12) float64 array (SConeProjection order),
        (n, 13) for cyl_cone_vec (SCylConeProjection order)."""
        n = self.dims.angles
        w = 13 if self.kind == _lib.GEOM_CYLCONE else 12
        buf = (ctypes.c_double * (w * n)).from_address(ctypes.addressof(self.views))
        return np.array(buf, dtype=np.float64).reshape(n, w)


class Geometry2D:
    """A normalised b2t_geom2d plus the view array it points to."""

    def __init__(self, vol_geom, proj_geom):
        lib = _lib.load()
        t = proj_geom['type']
        if t not in ('parallel', 'fanflat', 'parallel_vec', 'fanflat_vec'):
            raise AstraError(2, "2D projector needs a 2D projection geometry, got %r" % t)
        if is_3d_vol(vol_geom):
            raise AstraError(1, "2D projector needs a 2D volume geometry")
        self.kind = _lib.GEOM_FAN2D if t in ('fanflat', 'fanflat_vec') else _lib.GEOM_PAR2D
        na, ndet = proj_shape(proj_geom)
        views = (_lib.View2D * na)()
        if t == 'parallel':
            ang = np.ascontiguousarray(np.asarray(proj_geom['ProjectionAngles'], dtype=np.float32).ravel())
            _lib.check(lib.b2t_par_views(na, ndet, _f32(proj_geom['DetectorWidth']), _lib.ptr(ang), views))
        elif t == 'fanflat':
            ang = np.ascontiguousarray(np.asarray(proj_geom['ProjectionAngles'], dtype=np.float32).ravel())
            _lib.check(lib.b2t_fan_views(na, ndet, _f32(proj_geom['DistanceOriginSource']),
                                         _f32(proj_geom['DistanceOriginDetector']),
                                         _f32(proj_geom['DetectorWidth']), _lib.ptr(ang), views))
        else:
            vec = np.ascontiguousarray(np.asarray(proj_geom['Vectors'], dtype=np.float64))
            _lib.check(lib.b2t_vec_views2d(na, ndet, _lib.ptr(vec), views))
        o = vol_geom['option']
        vg = _lib.VolGeom2D(vol_geom['GridColCount'], vol_geom['GridRowCount'], _f32(o['WindowMinX']),
                            _f32(o['WindowMaxX']), _f32(o['WindowMinY']), _f32(o['WindowMaxY']))
        scale = ctypes.c_float(0.0)
        _lib.check(lib.b2t_normalize_views2d(ctypes.byref(vg), self.kind, na, views, ctypes.byref(scale)))
        self.views = views
        self.output_scale = scale.value
        self.dims = _lib.Dims2D(vol_geom['GridColCount'], vol_geom['GridRowCount'], na, ndet)
        self.c = _lib.Geom2D(self.kind, self.dims, scale.value, views)
        self.vol_shape = vol_shape(vol_geom)
        self.proj_shape = (na, ndet)

    def views_array(self):
        n = self.dims.angles
        buf = (ctypes.c_float * (6 * n)).from_address(ctypes.addressof(self.views))
        return np.array(buf, dtype=np.float32).reshape(n, 6)
