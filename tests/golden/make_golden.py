"""Generate golden vectors from the reference ASTRA Toolbox's own CUDA build.

Run on a machine with a GPU after `make -f oracle/ref.mk` has built
oracle/_ref/libastra_ref.so from the reference sources:

    python tests/golden/make_golden.py OUTDIR [NAME_SUBSTRING]

It writes one .npz per case (seeded inputs, the reference's normalised view
vectors and its output) that tests/test_oracle_golden.py compares the FP64
oracle against.  The committed fixtures in tests/golden/ were produced by this
script; the inputs are regenerated from the same seeds by the tests.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)


def vol_geom3(rows, cols, slices, window=None):
    g = {'GridRowCount': rows, 'GridColCount': cols, 'GridSliceCount': slices, 'option': {}}
    o = g['option']
    if window is None:
        window = (-cols / 2., cols / 2., -rows / 2., rows / 2., -slices / 2., slices / 2.)
    (o['WindowMinX'], o['WindowMaxX'], o['WindowMinY'], o['WindowMaxY'],
     o['WindowMinZ'], o['WindowMaxZ']) = window
    return g


def vol_geom2(rows, cols):
    return {'GridRowCount': rows, 'GridColCount': cols,
            'option': {'WindowMinX': -cols / 2., 'WindowMaxX': cols / 2.,
                       'WindowMinY': -rows / 2., 'WindowMaxY': rows / 2.}}


def input_volume(shape, seed):
    rng = np.random.default_rng(seed)
    v = rng.random(shape, dtype=np.float32)
    v[..., : shape[-1] // 3] += 1.0
    return v.astype(np.float32)


def input_proj(shape, seed):
    return np.random.default_rng(seed).random(shape, dtype=np.float32)


def cone_vec_vectors():
    rng = np.random.default_rng(5)
    vecs = []
    for i in range(9):
        t = 2 * np.pi * i / 9
        if i % 3 == 0:
            src = np.array([5 * np.cos(t), 5 * np.sin(t), -140.0])
            det = np.array([0.0, 0.0, 70.0])
            u = np.array([np.cos(t), np.sin(t), 0.0])
            v = np.array([-np.sin(t), np.cos(t), 0.0])
        else:
            src = np.array([-140 * np.sin(t), 140 * np.cos(t), 3.0])
            det = np.array([70 * np.sin(t), -70 * np.cos(t), -2.0])
            u = np.array([np.cos(t), np.sin(t), 0.02])
            v = np.array([0.01, 0.0, 1.0])
        u += rng.normal(0, 0.01, 3)
        vecs.append(np.concatenate([src, det, u, v]))
    return np.array(vecs)


def cyl_vectors():
    """cyl_cone_vec rows (src, detector centre, u, v, radius): a circular orbit
    on a cylinder centred at the source (radius SOD + ODD), plus views with the
    source on the z axis (cylinder axis along y), so every marching direction
    occurs."""
    sod, odd, rows = 80.0, 40.0, []
    for i in range(10):
        t = 2 * np.pi * i / 10 + 0.1
        src = np.array([np.sin(t) * sod, -np.cos(t) * sod, 1.5])
        det = np.array([-np.sin(t) * odd, np.cos(t) * odd, -0.5])
        u = np.array([np.cos(t), np.sin(t), 0.0]) * 1.1
        v = np.array([0.0, 0.0, 0.9])
        rows.append(np.concatenate([src, det, u, v, [sod + odd]]))
    for sgn in (1.0, -1.0):
        src = np.array([2.0, -1.0, -sgn * sod])
        det = np.array([0.0, 0.0, sgn * odd])
        u = np.array([1.2, 0.0, 0.0])
        v = np.array([0.0, 1.0, 0.0])
        rows.append(np.concatenate([src, det, u, v, [sod + odd]]))
    return np.array(rows)


def par_vec_vectors():
    """Nine parallel-beam views whose rays run mostly along z, x and y in turn,
    each tilted; detector centre, u and v per view (parallel3d_vec rows)."""
    rows = []
    for i in range(9):
        t = 2 * np.pi * i / 9
        if i % 3 == 0:
            ray = np.array([0.2 * np.cos(t), 0.3 * np.sin(t), 1.0])
        elif i % 3 == 1:
            ray = np.array([1.0, 0.25 * np.sin(t), 0.35])
        else:
            ray = np.array([0.3 * np.cos(t), -1.0, 0.4])
        ray /= np.linalg.norm(ray)
        a = np.array([0.0, 0.0, 1.0]) if abs(ray[2]) < 0.9 else np.array([1.0, 0.0, 0.0])
        u = np.cross(ray, a)
        u *= 0.9 / np.linalg.norm(u)
        v = np.cross(ray, u)
        v *= 1.1 / np.linalg.norm(v)
        det = np.array([0.5 * np.cos(t), -0.4, 0.3 * np.sin(t)])
        rows.append(np.concatenate([ray, det, u, v]))
    return np.array(rows)


def cases():
    ang24 = np.linspace(0, 2 * np.pi, 24, endpoint=False).astype(np.float32)
    ang15 = np.linspace(0, np.pi, 15, endpoint=False).astype(np.float32)
    cone = ('cone', vol_geom3(36, 40, 32),
            {'type': 'cone', 'DetectorSpacingX': 1.0, 'DetectorSpacingY': 1.0, 'DetectorRowCount': 40,
             'DetectorColCount': 48, 'ProjectionAngles': ang24, 'DistanceOriginSource': 150.0,
             'DistanceOriginDetector': 80.0})
    par = ('parallel3d', vol_geom3(28, 30, 20),
           {'type': 'parallel3d', 'DetectorSpacingX': 0.7, 'DetectorSpacingY': 1.3, 'DetectorRowCount': 30,
            'DetectorColCount': 50, 'ProjectionAngles': ang15})
    cvec = ('cone_vec', vol_geom3(30, 34, 28),
            {'type': 'cone_vec', 'DetectorRowCount': 38, 'DetectorColCount': 42, 'Vectors': cone_vec_vectors()})
    aniso = ('cone_aniso', vol_geom3(34, 30, 26, (-16.0, 18.0, -14.0, 16.0, -12.0, 14.0)),
             {'type': 'cone', 'DetectorSpacingX': 1.3, 'DetectorSpacingY': 0.8, 'DetectorRowCount': 36,
              'DetectorColCount': 44, 'ProjectionAngles': ang24 + 0.3, 'DistanceOriginSource': 120.0,
              'DistanceOriginDetector': 60.0})
    out = []
    for name, vg, pg in (cone, par, cvec, aniso):
        out.append(("fp3d_" + name, "fp3d", vg, pg, {}))
        out.append(("bp3d_" + name, "bp3d", vg, pg, {}))
    out.append(("fp3d_cone_ss2", "fp3d", cone[1], cone[2], {'rays': 2}))
    out.append(("bp3d_cone_ss2", "bp3d", cone[1], cone[2], {'rays': 2}))
    # 2d_weighting is meant for single-slice volumes: the reference launches it
    # with one z voxel per thread on a grid of ceil(nz / 6) blocks
    # (cuda/3d/cone_bp.cu:357-358), so on thicker volumes it fills only every
    # sixth slice
    out.append(("bp3d_cone_2dw", "bp3d", vol_geom3(36, 40, 1), cone[2], {'kernel': 3}))
    out.append(("bp3d_cone_fdkw", "bp3d", cone[1], cone[2], {'kernel': 2}))
    # sum_square_weights (parallel beams only): circular, and anisotropic
    # voxels with rays along each axis
    out.append(("fp3d_sumsqw_par", "sumsqw", par[1], par[2], {}))
    out.append(("fp3d_sumsqw_vec_aniso", "sumsqw", aniso[1],
                {'type': 'parallel3d_vec', 'DetectorRowCount': 36, 'DetectorColCount': 44,
                 'Vectors': par_vec_vectors()}, {}))
    # cyl_cone_vec: FP, voxel-driven BP, matched BP
    cyl = ('cyl', vol_geom3(34, 30, 28, (-15.0, 15.0, -17.0, 17.0, -14.0, 14.0)),
           {'type': 'cyl_cone_vec', 'DetectorRowCount': 40, 'DetectorColCount': 46, 'Vectors': cyl_vectors()})
    out.append(("cyl_fp", "cylfp", cyl[1], cyl[2], {}))
    out.append(("cyl_bp", "cylbp", cyl[1], cyl[2], {}))
    out.append(("cyl_bpm", "cylbpm", cyl[1], cyl[2], {}))
    ang72 = np.linspace(0, 2 * np.pi, 72, endpoint=False).astype(np.float32)
    fdkg = {'type': 'cone', 'DetectorSpacingX': 1.0, 'DetectorSpacingY': 1.0, 'DetectorRowCount': 40,
            'DetectorColCount': 56, 'ProjectionAngles': ang72, 'DistanceOriginSource': 200.0,
            'DistanceOriginDetector': 100.0}
    out.append(("fdk_cone", "fdk", vol_geom3(36, 36, 28), fdkg, {}))
    short = dict(fdkg)
    fan_half = np.arctan(56 * 0.5 / 300.0)
    short['ProjectionAngles'] = np.linspace(0, np.pi + 2 * fan_half, 60).astype(np.float32)
    out.append(("fdk_cone_short", "fdk", vol_geom3(36, 36, 28), short, {'short_scan': True}))
    ang2 = np.linspace(0, np.pi, 45, endpoint=False).astype(np.float32)
    angf = np.linspace(0, 2 * np.pi, 40, endpoint=False).astype(np.float32)
    par2 = {'type': 'parallel', 'DetectorWidth': 1.2, 'DetectorCount': 70, 'ProjectionAngles': ang2}
    fan2 = {'type': 'fanflat', 'DetectorWidth': 1.5, 'DetectorCount': 90, 'ProjectionAngles': angf,
            'DistanceOriginSource': 120.0, 'DistanceOriginDetector': 60.0}
    out.append(("fp2d_par", "fp2d", vol_geom2(48, 56), par2, {}))
    out.append(("bp2d_par", "bp2d", vol_geom2(48, 56), par2, {}))
    out.append(("fp2d_fan", "fp2d", vol_geom2(48, 56), fan2, {}))
    out.append(("bp2d_fan", "bp2d", vol_geom2(48, 56), fan2, {}))
    out.append(("bp2d_fan_fbp", "bp2d", vol_geom2(48, 56), fan2, {'fbp': True}))
    return out


def main(outdir, only=None):
    import torch
    from oracle import ref
    os.makedirs(outdir, exist_ok=True)
    for seed, (name, op, vg, pg, opt) in enumerate(cases()):
        if only and only not in name:
            continue
        if op in ("cylfp", "cylbp", "cylbpm"):
            views, vs = ref.geom3d(vg, pg)
            vshape = (vg['GridSliceCount'], vg['GridRowCount'], vg['GridColCount'])
            pshape = (pg['DetectorRowCount'], views.shape[0], pg['DetectorColCount'])
            if op == "cylfp":
                inp = input_volume(vshape, seed)
                res = ref.cuda_cyl('fp', views, torch.from_numpy(inp).cuda(), vshape, pshape[2], pshape[0], vs)
            else:
                inp = input_proj(pshape, seed)
                res = ref.cuda_cyl('bp' if op == "cylbp" else 'bp_matched', views, torch.from_numpy(inp).cuda(),
                                   vshape, pshape[2], pshape[0], vs)
            np.savez_compressed(os.path.join(outdir, name + ".npz"), views=views, vol_scale=vs, input=inp,
                                output=res.cpu().numpy(), kind=5)
            print("wrote", name)
            continue
        if op in ("fp3d", "bp3d", "fdk", "sumsqw"):
            views, vs = ref.geom3d(vg, pg)
            kind = 2 if pg['type'] in ('cone', 'cone_vec') else 1
            vshape = (vg['GridSliceCount'], vg['GridRowCount'], vg['GridColCount'])
            na = views.shape[0]
            pshape = (pg['DetectorRowCount'], na, pg['DetectorColCount'])
            if op == "sumsqw":
                res = ref.cuda_sumsqw(views, vshape, pshape[2], pshape[0], vs)
                np.savez_compressed(os.path.join(outdir, name + ".npz"), views=views, vol_scale=vs,
                                    vol_shape=np.array(vshape), input=np.zeros(0, np.float32),
                                    output=res.cpu().numpy(), kind=kind)
                print("wrote", name)
                continue
            if op == "fp3d":
                inp = input_volume(vshape, seed)
                res = ref.cuda_fp3d(kind, views, torch.from_numpy(inp).cuda(), pshape[2], pshape[0], vs,
                                    rays=opt.get('rays', 1))
            elif op == "bp3d":
                inp = input_proj(pshape, seed)
                res = ref.cuda_bp3d(kind, views, torch.from_numpy(inp).cuda(), vshape, vs,
                                    kernel=opt.get('kernel', 0), rays=opt.get('rays', 1))
            else:
                vol = input_volume(vshape, seed)
                inp = ref.cuda_fp3d(kind, views, torch.from_numpy(vol).cuda(), pshape[2], pshape[0], vs).cpu().numpy()
                res = ref.cuda_fdk(views, torch.from_numpy(inp.copy()).cuda(), vshape, vs,
                                   short_scan=opt.get('short_scan', False))
            np.savez_compressed(os.path.join(outdir, name + ".npz"), views=views, vol_scale=vs, input=inp,
                                output=res.cpu().numpy(), kind=kind)
        else:
            views, sc = ref.geom2d(vg, pg)
            kind = 4 if pg['type'] in ('fanflat', 'fanflat_vec') else 3
            vshape = (vg['GridRowCount'], vg['GridColCount'])
            na = views.shape[0]
            pshape = (na, pg['DetectorCount'])
            if op == "fp2d":
                inp = input_volume(vshape, seed)
                res = ref.cuda_fp2d(kind, views, torch.from_numpy(inp).cuda(), pshape[1], sc)
            else:
                inp = input_proj(pshape, seed)
                res = ref.cuda_bp2d(kind, views, torch.from_numpy(inp).cuda(), vshape, sc, fbp=opt.get('fbp', False))
            np.savez_compressed(os.path.join(outdir, name + ".npz"), views=views, out_scale=sc, input=inp,
                                output=res.cpu().numpy(), kind=kind)
        print("wrote", name)


if __name__ == "__main__":
    if len(sys.argv) < 2:
        sys.exit("usage: python tests/golden/make_golden.py OUTDIR [NAME_SUBSTRING]")
    main(sys.argv[1], sys.argv[2] if len(sys.argv) > 2 else None)
