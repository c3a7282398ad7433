"""The reference's own host code running on libb2tomo through the shim build
(oracle/ref_shim.mk: the reference compiled with its cuda/3d projector entry
points ConeFP / ConeBP / Par3DFP / Par3DBP replaced by calls into the C ABI,
oracle/ref_shim.cu, whose static_asserts check at compile time that
SConeProjection / SPar3DProjection / SDimensions3D have the layouts of
b2t_view3d / b2t_dims3d).

- Entry points: the reference's ConeFP / ConeBP / Par3DFP / Par3DBP through
  the shim give this library's results bit for bit.
- The reference's CompositeGeometryManager (astraCUDA3d::FP / BP dispatch):
  linked GPU data, the direct_FP3D path, equals host data, the
  create_sino3d_gpu path (the reference's tests/python/integration/
  test_dlpack3d.py:123-133), and a job split under a GPU memory limit equals
  the unsplit one (tests/python/functional/test_multigpu_consistency.py:
  39-52), for FP and BP.
- The reference's SIRT3D_CUDA object on the library reaches this library's
  own SIRT3D result (the same operators; 1e-5 after 10 iterations), and its
  FDK_CUDA (its weighting and cuFFT filter, the library's BP) stays within
  2e-3 of its all-texture FDK.
"""
import importlib

import numpy as np
import pytest

from conftest import rel_l2

torch = pytest.importorskip("torch")
ref = pytest.importorskip("oracle.ref")
pytestmark = pytest.mark.gpu

if not (ref.available() and ref.shim_available()):
    pytest.skip("the reference builds (oracle/_ref) are not built", allow_module_level=True)

N, NA, NU, NV, SOD, ODD = 64, 90, 96, 80, 200.0, 100.0


def _geom(astra):
    ang = np.linspace(0, 2 * np.pi, NA, endpoint=False).astype(np.float32)
    vg = astra.create_vol_geom(N, N, N)
    pg = astra.create_proj_geom('cone', 1.0, 1.0, NV, NU, ang, SOD, ODD)
    return ang, vg, pg


def _vol(seed=0):
    ph = importlib.import_module("astra-toolbox_b200.phantom")
    return ph.ellipsoids((N, N, N), 8, seed=seed, axes=(4.0, 24.0), device='cuda')


def test_shim_entry_points_are_the_library(astra):
    ang, vg, pg = _geom(astra)
    pr = astra.Projector3D(pg, vg)
    vol = _vol()
    ours = torch.zeros(pr.proj_shape, device='cuda')
    pr.fp(vol, ours)
    with ref.use_shim():
        views, vs = ref.geom3d(vg, pg)
        shim_fp = ref.cuda_fp3d(2, views, vol, NU, NV, vs)
        shim_bp = ref.cuda_bp3d(2, views, ours, (N, N, N), vs)
    assert torch.equal(shim_fp, ours)
    back = torch.zeros(pr.vol_shape, device='cuda')
    pr.bp(ours, back)
    assert torch.equal(shim_bp, back)
    # parallel beam through Par3DFP / Par3DBP
    pgp = astra.create_proj_geom('parallel3d', 1.0, 1.0, NV, NU, ang[:45] / 2)
    prp = astra.Projector3D(pgp, vg)
    op = torch.zeros(prp.proj_shape, device='cuda')
    prp.fp(vol, op)
    with ref.use_shim():
        views, vs = ref.geom3d(vg, pgp)
        sp = ref.cuda_fp3d(1, views, vol, NU, NV, vs)
    assert torch.equal(sp, op)


@pytest.mark.parametrize("op", ["fp", "bp"])
def test_shim_composite_manager_paths_agree(astra, op):
    ang, vg, pg = _geom(astra)
    pr = astra.Projector3D(pg, vg)
    vol = _vol(1)
    proj = torch.zeros(pr.proj_shape, device='cuda')
    pr.fp(vol, proj)
    ours = torch.zeros(pr.proj_shape if op == 'fp' else pr.vol_shape, device='cuda')
    if op == 'fp':
        pr.fp(vol, ours)
    else:
        pr.bp(proj, ours)
    with ref.use_shim():
        # direct_FP3D / direct_BP3D: linked device data
        p_lnk = torch.full(pr.proj_shape, 5.0, device='cuda') if op == 'fp' else proj.clone()
        v_lnk = vol.clone() if op == 'fp' else torch.full(pr.vol_shape, 5.0, device='cuda')
        ref.cgm_cone(op, ang, SOD, ODD, p_lnk, v_lnk)
        # create_sino3d_gpu / create_backprojection3d_gpu: host data
        p_host = np.zeros(pr.proj_shape, np.float32) if op == 'fp' else proj.cpu().numpy()
        v_host = vol.cpu().numpy() if op == 'fp' else np.zeros(pr.vol_shape, np.float32)
        ref.cgm_cone(op, ang, SOD, ODD, p_host, v_host, gpu_data=False)
        # the same under a memory limit below the job's size: split into pieces
        p_split = np.zeros(pr.proj_shape, np.float32) if op == 'fp' else proj.cpu().numpy()
        v_split = vol.cpu().numpy() if op == 'fp' else np.zeros(pr.vol_shape, np.float32)
        ref.cgm_cone(op, ang, SOD, ODD, p_split, v_split, memory=1_500_000, gpu_data=False)
    got_lnk = (p_lnk if op == 'fp' else v_lnk).cpu().numpy()
    got_host = p_host if op == 'fp' else v_host
    got_split = p_split if op == 'fp' else v_split
    want = ours.cpu().numpy()
    assert rel_l2(got_lnk, want) < 1e-6
    assert np.array_equal(got_host, got_lnk)
    assert rel_l2(got_split, got_host) < 1e-6


def test_shim_sirt3d_and_fdk_objects(astra):
    A = importlib.import_module("astra-toolbox_b200.algorithm")
    D3 = importlib.import_module("astra-toolbox_b200.data3d")
    ang, vg, pg = _geom(astra)
    pr = astra.Projector3D(pg, vg)
    vol = _vol(2)
    proj = torch.zeros(pr.proj_shape, device='cuda')
    pr.fp(vol, proj)
    # this library's SIRT3D
    pid = D3.link('-proj3d', pg, proj)
    rid = D3.create('-vol', vg, 0)
    cfg = A.astra_dict('SIRT3D_CUDA')
    cfg['ProjectionDataId'] = pid
    cfg['ReconstructionDataId'] = rid
    aid = A.create(cfg)
    A.run(aid, 10)
    ours = D3.get(rid)
    A.delete(aid)
    D3.delete([pid, rid])
    with ref.use_shim():
        x = torch.zeros(pr.vol_shape, device='cuda')
        alg = ref.Algo3D('SIRT3D_CUDA', ang, SOD, ODD, proj, x)
        alg.run(10)
        alg.close()
        f_shim = torch.zeros(pr.vol_shape, device='cuda')
        alg = ref.Algo3D('FDK_CUDA', ang, SOD, ODD, proj.clone(), f_shim)
        alg.run(1)
        alg.close()
    assert rel_l2(x.cpu().numpy(), ours) < 1e-5
    f_ref = torch.zeros(pr.vol_shape, device='cuda')
    alg = ref.Algo3D('FDK_CUDA', ang, SOD, ODD, proj.clone(), f_ref)
    alg.run(1)
    alg.close()
    # the reference's texture BP weights with 8-bit fractions (measured 3.3e-4
    # here); the stated tolerance against the reference build is 2e-3
    assert rel_l2(f_shim.cpu().numpy(), f_ref.cpu().numpy()) < 2e-3
