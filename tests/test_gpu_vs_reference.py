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


@pytest.mark.parametrize("idx", range(21))
def test_case_vs_reference_cuda(astra, idx):
    ref = _ref()
    mg, cases = _cases()
    if idx >= len(cases):
        pytest.skip("no such case")
    name, op, vg, pg, opt = cases[idx]
    P = importlib.import_module("astra-toolbox_b200.projector")
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
