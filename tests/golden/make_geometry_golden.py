"""Generate per-view geometry fixtures from the reference's own
convertAstraGeometry (built from its sources into oracle/_ref by oracle/ref.mk).

    python tests/golden/make_geometry_golden.py

Writes tests/golden/geometry_views.npz: for each case in CASES, the reference's
normalised view vectors and voxel size / output scale.  Host code only: runs
without a GPU.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)


def cases():
    rng = np.random.Generator(np.random.PCG64(1))
    ang = np.sort(rng.uniform(0, 2 * np.pi, 37)).astype(np.float32)
    V = rng.normal(size=(29, 12))
    V2 = rng.normal(size=(11, 6))
    # cyl_cone_vec rows: 12 vector components and a positive radius
    V13 = rng.normal(size=(17, 13))
    V13[:, 12] = np.abs(V13[:, 12]) * 50.0 + 100.0
    vg3 = {'GridRowCount': 48, 'GridColCount': 40, 'GridSliceCount': 32,
           'option': {'WindowMinX': -21.3, 'WindowMaxX': 19.1, 'WindowMinY': -25.7, 'WindowMaxY': 22.9,
                      'WindowMinZ': -13.2, 'WindowMaxZ': 18.4}}
    vg2 = {'GridRowCount': 64, 'GridColCount': 64,
           'option': {'WindowMinX': -30.5, 'WindowMaxX': 33.5, 'WindowMinY': -31.0, 'WindowMaxY': 33.0}}
    c3 = [
        ('cone', vg3, {'type': 'cone', 'DetectorSpacingX': 1.3, 'DetectorSpacingY': 0.9, 'DetectorRowCount': 50,
                       'DetectorColCount': 60, 'ProjectionAngles': ang, 'DistanceOriginSource': 700.5,
                       'DistanceOriginDetector': 300.25}),
        ('parallel3d', vg3, {'type': 'parallel3d', 'DetectorSpacingX': 1.1, 'DetectorSpacingY': 0.7,
                             'DetectorRowCount': 50, 'DetectorColCount': 60, 'ProjectionAngles': ang}),
        ('cone_vec', vg3, {'type': 'cone_vec', 'DetectorRowCount': 50, 'DetectorColCount': 60, 'Vectors': V}),
        ('parallel3d_vec', vg3, {'type': 'parallel3d_vec', 'DetectorRowCount': 50, 'DetectorColCount': 60,
                                 'Vectors': V}),
        ('cyl_cone_vec', vg3, {'type': 'cyl_cone_vec', 'DetectorRowCount': 50, 'DetectorColCount': 60,
                               'Vectors': V13}),
    ]
    c2 = [
        ('parallel', vg2, {'type': 'parallel', 'DetectorWidth': 1.3, 'DetectorCount': 90, 'ProjectionAngles': ang}),
        ('fanflat', vg2, {'type': 'fanflat', 'DetectorWidth': 1.3, 'DetectorCount': 90, 'ProjectionAngles': ang,
                          'DistanceOriginSource': 400.5, 'DistanceOriginDetector': 200.25}),
        ('parallel_vec', vg2, {'type': 'parallel_vec', 'DetectorCount': 90, 'Vectors': V2}),
        ('fanflat_vec', vg2, {'type': 'fanflat_vec', 'DetectorCount': 90, 'Vectors': V2}),
    ]
    return c3, c2


def main(out):
    from oracle import ref
    c3, c2 = cases()
    arrays = {}
    for name, vg, pg in c3:
        views, vs = ref.geom3d(vg, pg)
        arrays[name + "_views"] = views
        arrays[name + "_scale"] = vs
    for name, vg, pg in c2:
        views, sc = ref.geom2d(vg, pg)
        arrays[name + "_views"] = views
        arrays[name + "_scale"] = np.array([sc], dtype=np.float32)
    np.savez(out, **arrays)
    print("wrote", out)


if __name__ == "__main__":
    main(os.path.join(os.path.dirname(os.path.abspath(__file__)), "geometry_views.npz"))
