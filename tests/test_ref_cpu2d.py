"""The reference's own CPU 2D projectors (its CPU-only build, oracle/ref_cpu.mk)
against the FP64 oracle (CPU) and against the library's 2D CUDA path (GPU).

Models and stated tolerances (relative L2 on seeded ellipse phantoms of the
C1 shape, 256^2, 180 views over pi, 384 detectors; fan beam at 128^2):
- 'linear' (src/ParallelBeamLinearKernelProjector2D.cpp) samples the same
  linear-interpolation model as the CUDA projector (the reference's own test,
  tests/python/functional/test_line2d.py:476-513, checks both against one
  analytic line integral): FP within 1e-4 (measured about 2e-5; the CPU code
  accumulates its weights in float32).  Its BP is the exact transpose of its
  FP, not the CUDA path's voxel-driven BP: within 2e-2.
- 'line' and 'strip' (and their fan-beam forms) discretise the same line
  integral differently: FP within 3e-2.
"""
import importlib

import numpy as np
import pytest

from conftest import rel_l2

ref = pytest.importorskip("oracle.ref")
if not ref.cpu_available():
    pytest.skip("the reference's CPU build (oracle/_ref/libastra_ref_cpu.so) is not built", allow_module_level=True)


def _phantom(n, seed=0):
    """10 seeded ellipses (the C1 phantom), numpy only."""
    rng = np.random.Generator(np.random.PCG64(seed))
    y, x = np.mgrid[0:n, 0:n] + 0.5 - n / 2
    img = np.zeros((n, n), dtype=np.float64)
    for _ in range(10):
        cx, cy = rng.uniform(-0.4, 0.4, 2) * n
        a, b = rng.uniform(10 * n / 256, 80 * n / 256, 2)
        t = rng.uniform(0, np.pi)
        xr = (x - cx) * np.cos(t) + (y - cy) * np.sin(t)
        yr = -(x - cx) * np.sin(t) + (y - cy) * np.cos(t)
        img[(xr / a) ** 2 + (yr / b) ** 2 <= 1] += rng.uniform(0, 1)
    return img.astype(np.float32)


def _par_setup(n=256, na=180, nd=384):
    ang = np.linspace(0, np.pi, na, endpoint=False).astype(np.float32)
    vg = {'GridRowCount': n, 'GridColCount': n,
          'option': {'WindowMinX': -n / 2., 'WindowMaxX': n / 2., 'WindowMinY': -n / 2., 'WindowMaxY': n / 2.}}
    pg = {'type': 'parallel', 'DetectorWidth': 1.0, 'DetectorCount': nd, 'ProjectionAngles': ang}
    return ang, vg, pg


def test_oracle_matches_reference_cpu_linear(orc):
    """The oracle's 2D parallel FP (the CUDA model in FP64) equals the
    reference's CPU 'linear' projector up to the latter's float32 rounding."""
    if not ref.available():
        pytest.skip("reference build (geometry conversion) not built")
    ang, vg, pg = _par_setup()
    vol = _phantom(256)
    views, sc = ref.geom2d(vg, pg)
    o = orc.par_fp(views, vol, 384, sc)
    lin = ref.cpu_fp2d('parallel', 'linear', vol, ang, 384)
    assert rel_l2(o, lin) < 1e-4
    for kernel, tol in (('line', 3e-2), ('strip', 3e-2)):
        assert rel_l2(o, ref.cpu_fp2d('parallel', kernel, vol, ang, 384)) < tol, kernel


@pytest.mark.gpu
def test_cuda_2d_vs_reference_cpu_projectors(astra):
    import torch
    ang, _, _ = _par_setup()
    vg = astra.create_vol_geom(256, 256)
    pg = astra.create_proj_geom('parallel', 1.0, 384, ang)
    pr = astra.Projector2D(pg, vg)
    vol = _phantom(256)
    sino = torch.zeros(pr.proj_shape, device='cuda')
    pr.fp(torch.from_numpy(vol).cuda(), sino)
    got = sino.cpu().numpy()
    lin = ref.cpu_fp2d('parallel', 'linear', vol, ang, 384)
    assert rel_l2(got, lin) < 1e-4
    for kernel in ('line', 'strip'):
        assert rel_l2(got, ref.cpu_fp2d('parallel', kernel, vol, ang, 384)) < 3e-2, kernel
    back = torch.zeros(pr.vol_shape, device='cuda')
    pr.bp(torch.from_numpy(lin).cuda(), back)
    assert rel_l2(back.cpu().numpy(), ref.cpu_bp2d('parallel', 'linear', lin, (256, 256), ang)) < 2e-2


@pytest.mark.gpu
def test_cuda_fan_vs_reference_cpu_projectors(astra):
    import torch
    n, na, nd = 128, 90, 192
    ang = np.linspace(0, 2 * np.pi, na, endpoint=False).astype(np.float32)
    vg = astra.create_vol_geom(n, n)
    pg = astra.create_proj_geom('fanflat', 1.0, nd, ang, 2.0 * n, 1.0 * n)
    pr = astra.Projector2D(pg, vg)
    vol = _phantom(n, 1)
    sino = torch.zeros(pr.proj_shape, device='cuda')
    pr.fp(torch.from_numpy(vol).cuda(), sino)
    got = sino.cpu().numpy()
    for kernel in ('line', 'strip'):
        cpu = ref.cpu_fp2d('fanflat', kernel, vol, ang, nd, 1.0, 2.0 * n, 1.0 * n)
        assert rel_l2(got, cpu) < 3e-2, kernel


@pytest.mark.gpu
def test_cuda_sirt2d_vs_reference_cpu_sirt(astra):
    """SIRT 100 (C1): the CUDA SIRT and the reference's CPU SIRT with its
    'linear' projector reach reconstructions within 2e-2 of each other (their
    BPs differ: voxel-driven vs exact transpose) and the same residual
    within 10 %."""
    import torch
    A = importlib.import_module("astra-toolbox_b200.algorithm")
    D2 = importlib.import_module("astra-toolbox_b200.data2d")
    ang, _, _ = _par_setup()
    vg = astra.create_vol_geom(256, 256)
    pg = astra.create_proj_geom('parallel', 1.0, 384, ang)
    vol = _phantom(256)
    b = ref.cpu_fp2d('parallel', 'linear', vol, ang, 384)
    sid = D2.link('-sino', pg, torch.from_numpy(b).cuda())
    rid = D2.create('-vol', vg, 0)
    cfg = A.astra_dict('SIRT_CUDA')
    cfg['ProjectionDataId'] = sid
    cfg['ReconstructionDataId'] = rid
    aid = A.create(cfg)
    A.run(aid, 100)
    got = D2.get(rid)
    A.delete(aid)
    D2.delete([sid, rid])
    cpu = ref.cpu_sirt2d('parallel', 'linear', b, (256, 256), ang, 100)
    assert rel_l2(got, cpu) < 2e-2
    r_gpu = np.linalg.norm(ref.cpu_fp2d('parallel', 'linear', got, ang, 384) - b)
    r_cpu = np.linalg.norm(ref.cpu_fp2d('parallel', 'linear', cpu, ang, 384) - b)
    assert abs(r_gpu - r_cpu) < 0.1 * r_cpu
