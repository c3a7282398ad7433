"""libb2tomo against the reference's own CUDA build on the same inputs, on the
GPU (needs oracle/_ref/libastra_ref.so, built from the reference sources by
oracle/ref.mk).  Bar: 2e-3 relative L2 (the reference interpolates with 8-bit
texture weights)."""
import importlib
import os
import sys

import numpy as np
import pytest

from conftest import rel_l2

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))


def _ref():
    from oracle import ref
    if not ref.available():
        pytest.skip("reference build not present")
    return ref


def _cases():
    mg = importlib.import_module("make_golden")
    return mg, [c for c in mg.cases()]


@pytest.mark.parametrize("idx", range(24))
def test_case_vs_reference_cuda(astra, idx):
    ref = _ref()
    mg, cases = _cases()
    if idx >= len(cases):
        pytest.skip("no such case")
    name, op, vg, pg, opt = cases[idx]
    P = importlib.import_module("astra-toolbox_b200.projector")
    if op in ("cylfp", "cylbp", "cylbpm"):
        opts = {'ProjectionKernel': 'matched_bp'} if op == "cylbpm" else {}
        pr = P.Projector3D(pg, vg, opts)
        views, vs = pr.geom.views_array(), pr.geom.vol_scale
        nv, na, nu = pr.proj_shape
        if op == "cylfp":
            inp = torch.from_numpy(mg.input_volume(pr.vol_shape, idx)).cuda()
            want = ref.cuda_cyl('fp', views, inp, pr.vol_shape, nu, nv, vs)
            got = torch.zeros(pr.proj_shape, device='cuda')
            pr.fp(inp, got)
        else:
            inp = torch.from_numpy(mg.input_proj(pr.proj_shape, idx)).cuda()
            want = ref.cuda_cyl('bp' if op == "cylbp" else 'bp_matched', views, inp, pr.vol_shape, nu, nv, vs)
            got = torch.zeros(pr.vol_shape, device='cuda')
            pr.bp(inp, got)
        err = rel_l2(got.cpu().numpy(), want.cpu().numpy())
        assert err < (1e-4 if op == "cylbpm" else 2e-3), (name, err)
        return
    if op == "sumsqw":
        pr = P.Projector3D(pg, vg, {'ProjectionKernel': 'sum_square_weights'})
        nv, na, nu = pr.proj_shape
        want = ref.cuda_sumsqw(pr.geom.views_array(), pr.vol_shape, nu, nv, pr.geom.vol_scale)
        got = torch.zeros(pr.proj_shape, device='cuda')
        pr.fp(torch.zeros(pr.vol_shape, device='cuda'), got)
        # no texture weights in this kernel: the bar is the float stepping
        err = rel_l2(got.cpu().numpy(), want.cpu().numpy())
        assert err < 1e-4, (name, err)
        return
    if op in ("fp3d", "bp3d", "fdk"):
        opts = {}
        if opt.get('rays'):
            opts = {'DetectorSuperSampling': opt['rays'], 'VoxelSuperSampling': opt['rays']}
        if opt.get('kernel') == 3:
            opts['ProjectionKernel'] = '2d_weighting'
        if opt.get('kernel') == 2:
            opts['ProjectionKernel'] = 'fdk_weighting'
        pr = P.Projector3D(pg, vg, opts)
        views = pr.geom.views_array()
        kind = pr.geom.kind
        nv, na, nu = pr.proj_shape
        if op == "fp3d":
            inp = torch.from_numpy(mg.input_volume(pr.vol_shape, idx)).cuda()
            want = ref.cuda_fp3d(kind, views, inp, nu, nv, pr.geom.vol_scale, rays=opt.get('rays', 1))
            got = torch.zeros(pr.proj_shape, device='cuda')
            pr.fp(inp, got)
        elif op == "bp3d":
            inp = torch.from_numpy(mg.input_proj(pr.proj_shape, idx)).cuda()
            want = ref.cuda_bp3d(kind, views, inp, pr.vol_shape, pr.geom.vol_scale, kernel=opt.get('kernel', 0),
                                 rays=opt.get('rays', 1))
            got = torch.zeros(pr.vol_shape, device='cuda')
            pr.bp(inp, got)
        else:
            vol = torch.from_numpy(mg.input_volume(pr.vol_shape, idx)).cuda()
            proj = torch.zeros(pr.proj_shape, device='cuda')
            pr.fp(vol, proj)
            want = ref.cuda_fdk(views, proj.clone(), pr.vol_shape, pr.geom.vol_scale,
                                short_scan=opt.get('short_scan', False))
            got = torch.zeros(pr.vol_shape, device='cuda')
            P.fdk(pr, proj, got, short_scan=opt.get('short_scan', False))
    else:
        pr = P.Projector2D(pg, vg)
        kind = pr.geom.kind
        views = pr.geom.views_array()
        if op == "fp2d":
            inp = torch.from_numpy(mg.input_volume(pr.vol_shape, idx)).cuda()
            want = ref.cuda_fp2d(kind, views, inp, pr.proj_shape[1], pr.geom.output_scale)
            got = torch.zeros(pr.proj_shape, device='cuda')
            pr.fp(inp, got)
        else:
            inp = torch.from_numpy(mg.input_proj(pr.proj_shape, idx)).cuda()
            want = ref.cuda_bp2d(kind, views, inp, pr.vol_shape, pr.geom.output_scale, fbp=opt.get('fbp', False))
            got = torch.zeros(pr.vol_shape, device='cuda')
            pr.bp(inp, got, fbp_weight=opt.get('fbp', False))
    err = rel_l2(got.cpu().numpy(), want.cpu().numpy())
    assert err < 2e-3, (name, err)


@pytest.mark.parametrize("geom", ["parallel", "fanflat"])
def test_sart2d_vs_reference_cuda(astra, orc, geom):
    """SART_CUDA against the reference's own CCudaSartAlgorithm (sequential
    order, relaxation 1), one sweep from zero.  The reference interpolates with
    8-bit texture weights: the oracle's tex8 mode tracks it within 2e-3, and
    libb2tomo (exact weights) within 5e-3."""
    ref = _ref()
    if geom == "parallel":
        ang = np.linspace(0, np.pi, 60, endpoint=False).astype(np.float32)
        vg = astra.create_vol_geom(40, 44)
        pg = astra.create_proj_geom('parallel', 1.0, 64, ang)
    else:
        ang = np.linspace(0, 2 * np.pi, 50, endpoint=False).astype(np.float32)
        vg = astra.create_vol_geom(36, 40)
        pg = astra.create_proj_geom('fanflat', 1.2, 70, ang, 110.0, 50.0)
    P = importlib.import_module("astra-toolbox_b200.projector")
    pr = P.Projector2D(pg, vg)
    views, sc = pr.geom.views_array(), pr.geom.output_scale
    kind = pr.geom.kind
    fp = orc.par_fp if kind == 3 else orc.fan_fp
    x_true = np.random.default_rng(9).random(pr.vol_shape).astype(np.float32)
    b = fp(views, x_true, pr.proj_shape[1], sc).astype(np.float32)
    iters = pr.proj_shape[0]
    want = ref.sart2d(vg, pg, b, np.zeros(pr.vol_shape, np.float32), iters)
    tex8 = orc.sart2d(kind, views, b, np.zeros(pr.vol_shape), sc, iters, tex8=True)
    assert rel_l2(tex8, want) < 2e-3, rel_l2(tex8, want)
    sid = astra.data2d.create('-sino', pg, b)
    rid = astra.data2d.create('-vol', vg, 0)
    cfg = astra.astra_dict('SART_CUDA')
    cfg['ProjectionDataId'] = sid
    cfg['ReconstructionDataId'] = rid
    cfg['option'] = {'ProjectionOrder': 'sequential'}
    aid = astra.algorithm.create(cfg)
    astra.algorithm.run(aid, iters)
    got = astra.data2d.get(rid)
    astra.algorithm.delete(aid)
    astra.data2d.delete([sid, rid])
    assert rel_l2(got, want) < 5e-3, rel_l2(got, want)
