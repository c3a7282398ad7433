"""Streamed projection of host-resident data (b2t_fp3d_host, b2t_bp3d_host,
b2t_fdk_host): the split plan on CPU, and on the GPU the reference's
memory-limited consistency pattern (tests/python/functional/
test_multigpu_consistency.py:39-52: a memory budget set with set_gpu_index
must not change the results)."""
import ctypes
import importlib

import numpy as np
import pytest

from conftest import rel_l2

torch = pytest.importorskip("torch")


def _geom(astra, n=96, na=96, short=False):
    ang = np.linspace(0, 2 * np.pi, na, endpoint=False).astype(np.float32)
    if short:
        fan = np.arctan(n * 0.5 / (10.0 * n))
        ang = np.linspace(0, np.pi + 2 * fan, na).astype(np.float32)
    vg = astra.create_vol_geom(n, n, n)
    pg = astra.create_proj_geom('cone', 1.0, 1.0, n, n, ang, 4.0 * n, 2.0 * n)
    return vg, pg


def _plan(lib, geom, op, budget):
    dev = (ctypes.c_int32 * 1)(0)
    L = importlib.import_module("astra-toolbox_b200._lib")
    cfg = L.StreamConfig(budget, 1, ctypes.cast(dev, ctypes.POINTER(ctypes.c_int32)))
    slab, block = ctypes.c_uint32(0), ctypes.c_uint32(0)
    st = lib.b2t_stream_plan(op, ctypes.byref(geom.c), ctypes.byref(cfg), ctypes.byref(slab), ctypes.byref(block))
    return st, slab.value, block.value


def test_stream_plan_splits_by_budget(astra, geo):
    """The split follows the budget: the whole volume in one slab when it
    fits, with angle blocks of at most an eighth of the views (at least 16)
    so that transfers overlap compute; thinner slabs and smaller blocks when
    it does not fit, and an error below one slice/view."""
    lib = importlib.import_module("astra-toolbox_b200._lib").load()
    vg, pg = _geom(astra)
    g = geo.Geometry3D(vg, pg)
    st, z, a = _plan(lib, g, 0, 1 << 40)
    assert st == 0 and (z, a) == (96, 16)
    st, z, a = _plan(lib, g, 0, 8_000_000)
    assert st == 0 and 1 <= z < 96 and 1 <= a < 96
    for op in (1, 2):
        st, z2, a2 = _plan(lib, g, op, 8_000_000)
        assert st == 0 and 1 <= z2 <= 96 and 1 <= a2 < 96
    st, _, _ = _plan(lib, g, 0, 1000)
    assert st != 0


@pytest.mark.gpu
def test_memory_budget_keeps_results(astra):
    """FP, BP, FDK (full and short scan) and accumulate under an 8 MB budget
    (host-resident data, many slabs and angle blocks) equal the unsplit
    device-resident results up to float summation order."""
    P = importlib.import_module("astra-toolbox_b200.projector")
    vg, pg = _geom(astra)
    phantom = importlib.import_module("astra-toolbox_b200.phantom")
    pr = P.Projector3D(pg, vg)
    vol = phantom.ellipsoids(pr.vol_shape, 8, seed=1, axes=(5.0, 30.0), device='cpu').numpy()
    try:
        sid, p_single = astra.create_sino3d_gpu(vol, pg, vg)
        astra.data3d.delete(sid)
        vid, b_single = astra.create_backprojection3d_gpu(p_single, pg, vg)
        astra.data3d.delete(vid)
        pid = astra.create_projector('cuda3d', pg, vg)
        W = astra.OpTomo(pid)
        r_single = W.reconstruct('FDK_CUDA', p_single)
        astra.set_gpu_index(0, memory=8_000_000)
        z, a = P.stream_plan(pr, 'fp')
        assert z < 96 and a < 96
        sid, p_multi = astra.create_sino3d_gpu(vol, pg, vg)
        assert not astra.data3d.get_shared(sid).is_cuda  # host-resident, streamed
        astra.data3d.delete(sid)
        assert rel_l2(p_multi, p_single) < 1e-5
        assert np.allclose(p_multi, p_single, rtol=1e-3, atol=1e-1)
        vid, b_multi = astra.create_backprojection3d_gpu(p_single, pg, vg)
        astra.data3d.delete(vid)
        assert rel_l2(b_multi, b_single) < 1e-5
        r_multi = W.reconstruct('FDK_CUDA', p_single)
        assert rel_l2(r_multi, r_single) < 1e-5
        assert np.allclose(r_multi, r_single, rtol=1e-3, atol=1e-3)
        # accumulate_FP adds onto the host-resident projections
        v_id = astra.data3d.create('-vol', vg, vol)
        p_id = astra.data3d.create('-sino', pg, 1.0)
        astra.experimental.accumulate_FP(pid, v_id, p_id)
        assert rel_l2(astra.data3d.get(p_id), p_single + 1.0) < 1e-5
        astra.data3d.delete([v_id, p_id])
    finally:
        astra.set_gpu_index(0, memory=0)
    # short-scan FDK: Parker weights of the whole scan in every angle block
    vg2, pg2 = _geom(astra, short=True)
    sid, p2 = astra.create_sino3d_gpu(vol, pg2, vg2)
    astra.data3d.delete(sid)
    pid2 = astra.create_projector('cuda3d', pg2, vg2)
    W2 = astra.OpTomo(pid2)
    want = W2.reconstruct('FDK_CUDA', p2, extraOptions={'ShortScan': True})
    try:
        astra.set_gpu_index(0, memory=8_000_000)
        got = W2.reconstruct('FDK_CUDA', p2, extraOptions={'ShortScan': True})
    finally:
        astra.set_gpu_index(0, memory=0)
    assert rel_l2(got, want) < 1e-5


@pytest.mark.gpu
def test_host_entry_points_whole_volume(astra):
    """With no budget the whole volume fits: the streamed FP lays the volume
    out in cells once and projects it in angle blocks (an eighth of the views
    each), the streamed BP uploads angle blocks while it computes.  The FP
    equals the device FP exactly (every ray is computed by the same kernel);
    the BP equals it up to the order in which the blocks are summed."""
    import torch
    P = importlib.import_module("astra-toolbox_b200.projector")
    phantom = importlib.import_module("astra-toolbox_b200.phantom")
    vg, pg = _geom(astra)
    pr = P.Projector3D(pg, vg)
    astra.set_gpu_index(0, memory=0)
    z, a = P.stream_plan(pr, 'fp')
    assert z == pr.vol_shape[0] and a == 16  # one slab, 96 views in blocks of 16
    vol = phantom.ellipsoids(pr.vol_shape, 8, seed=2, axes=(5.0, 30.0), device='cuda')
    dproj = torch.zeros(pr.proj_shape, device='cuda')
    pr.fp(vol, dproj)
    hvol = vol.cpu().pin_memory()
    hproj = torch.zeros(pr.proj_shape).pin_memory()
    P.fp3d_host(pr, hvol, hproj)
    assert torch.equal(hproj, dproj.cpu())
    drec = torch.zeros(pr.vol_shape, device='cuda')
    pr.bp(dproj, drec)
    hrec = torch.zeros(pr.vol_shape).pin_memory()
    P.bp3d_host(pr, hproj, hrec)
    assert rel_l2(hrec.numpy(), drec.cpu().numpy()) < 1e-6
    # accumulate onto the host arrays
    P.fp3d_host(pr, hvol, hproj, mode=0)
    assert rel_l2(hproj.numpy(), 2 * dproj.cpu().numpy()) < 1e-6
