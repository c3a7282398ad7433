"""Batched 3D problems (b2t_batch3d_*): one persistent launch per operation for
a mixed batch of parallel3d / parallel3d_vec / cone / cone_vec problems of
different sizes, view counts and detector supersampling, against the
single-problem direct-load projectors (B2T_SIMPLE_FP / B2T_SIMPLE_BP: the
same arithmetic, so bit for bit) and the FP64 oracle (1e-5 relative L2)."""
import importlib

import numpy as np
import pytest

from conftest import rel_l2

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _vec(n, rng, cone):
    vecs = []
    for i in range(n):
        t = 2 * np.pi * i / n
        if i % 3 == 0:
            # source mostly along z: z-major marching
            src = np.array([5 * np.cos(t), 5 * np.sin(t), -140.0])
            det = np.array([0.0, 0.0, 70.0])
            u = np.array([np.cos(t), np.sin(t), 0.0])
            v = np.array([-np.sin(t), np.cos(t), 0.0])
        else:
            src = np.array([-140 * np.sin(t), 140 * np.cos(t), 3.0])
            det = np.array([70 * np.sin(t), -70 * np.cos(t), -2.0])
            u = np.array([np.cos(t), np.sin(t), 0.02])
            v = np.array([0.01, 0.0, 1.0])
        u = u + rng.normal(0, 0.01, 3)
        if not cone:
            src = det - src
            src = src / np.linalg.norm(src)
        vecs.append(np.concatenate([src, det, u, v]))
    return np.array(vecs)


def _problems(astra):
    rng = np.random.default_rng(3)
    ang = np.linspace(0, 2 * np.pi, 30, endpoint=False).astype(np.float32)
    return [
        (astra.create_proj_geom('cone', 1.0, 1.0, 40, 48, ang, 150.0, 80.0), astra.create_vol_geom(36, 40, 32), {}),
        (astra.create_proj_geom('parallel3d', 1.0, 1.0, 24, 30, ang[:13] / 2), astra.create_vol_geom(28, 20, 22), {}),
        (astra.create_proj_geom('cone_vec', 38, 42, _vec(9, rng, True)), astra.create_vol_geom(34, 30, 28), {}),
        (astra.create_proj_geom('parallel3d_vec', 38, 42, _vec(7, rng, False)), astra.create_vol_geom(34, 30, 28),
         {}),
        (astra.create_proj_geom('cone', 1.3, 0.8, 18, 20, ang[:11] + 0.3, 120.0, 60.0),
         astra.create_vol_geom(16, 18, 9, -9.0, 9.0, -8.0, 8.0, -5.0, 4.0), {'DetectorSuperSampling': 2}),
        (astra.create_proj_geom('cone', 1.0, 1.0, 8, 12, ang[:5], 100.0, 50.0), astra.create_vol_geom(7, 5, 3), {}),
    ]


def _phantoms(batch, seed=1):
    rng = np.random.default_rng(seed)
    return [torch.from_numpy(rng.random(sh, dtype=np.float32)).cuda() for sh in batch.vol_shapes]


def test_batched_fp_bp_match_single_problem(astra, orc, monkeypatch):
    L = importlib.import_module("astra-toolbox_b200._lib")
    lib = L.load()
    probs = _problems(astra)
    B = astra.Batch3D(probs)
    vols = B.pack_vols(_phantoms(B))
    n0 = lib.b2t_kernel_launches()
    projs = B.fp(vols)
    torch.cuda.synchronize()
    assert lib.b2t_kernel_launches() - n0 == 1, "one persistent launch for the whole batch"
    n0 = lib.b2t_kernel_launches()
    back = B.bp(projs)
    torch.cuda.synchronize()
    assert lib.b2t_kernel_launches() - n0 == 1
    monkeypatch.setenv("B2T_SIMPLE_FP", "1")
    monkeypatch.setenv("B2T_SIMPLE_BP", "1")
    for i, (pg, vg, opts) in enumerate(probs):
        pr = astra.Projector3D(pg, vg, opts)
        v = B.vol_views(vols)[i].contiguous()
        p1 = torch.zeros(pr.proj_shape, device='cuda')
        pr.fp(v, p1)
        pb = B.proj_views(projs)[i]
        assert torch.equal(pb, p1), i
        b1 = torch.zeros(pr.vol_shape, device='cuda')
        pr.bp(pb.contiguous(), b1)
        assert torch.equal(B.vol_views(back)[i], b1), i
        kind = 2 if pr.geom.kind == 2 else 1
        rays = opts.get('DetectorSuperSampling', 1)
        nv, na, nu = pr.proj_shape
        ref = orc.fp3d(kind, pr.geom.views_array(), v.cpu().numpy(), nu, nv, pr.geom.vol_scale, rays=rays)
        assert rel_l2(pb.cpu().numpy(), ref) < 1e-5, i
        refb = orc.bp3d(kind, pr.geom.views_array(), pb.cpu().numpy(), pr.vol_shape, pr.geom.vol_scale)
        assert rel_l2(B.vol_views(back)[i].cpu().numpy(), refb) < 1e-5, i
    # accumulate mode adds
    p2 = projs.clone()
    B.fp(vols, p2, mode=L.MODE_ADD)
    assert torch.allclose(p2, 2 * projs, rtol=1e-6, atol=1e-6)
    b2 = back.clone()
    B.bp(projs, b2, mode=L.MODE_ADD)
    assert torch.allclose(b2, 2 * back, rtol=1e-6, atol=1e-5)
    B.close()


def test_batch_of_identical_problems_is_a_leading_dimension(astra):
    """Identical problems pack back to back, so a [B, z, y, x] tensor is the
    packed volume buffer as it is."""
    ang = np.linspace(0, np.pi, 16, endpoint=False).astype(np.float32)
    pg = astra.create_proj_geom('parallel3d', 1.0, 1.0, 16, 24, ang)
    vg = astra.create_vol_geom(16, 16, 8)
    B = astra.Batch3D([(pg, vg)] * 5)
    assert B.vol_offsets == [i * 16 * 16 * 8 for i in range(5)]
    assert B.proj_offsets == [i * 16 * 16 * 24 for i in range(5)]
    x = torch.rand(5, 8, 16, 16, device='cuda')
    p = B.fp(x.view(-1)).view(5, 16, 16, 24)
    pr = astra.Projector3D(pg, vg)
    for i in range(5):
        q = torch.zeros(pr.proj_shape, device='cuda')
        pr.fp(x[i].contiguous(), q)
        assert rel_l2(p[i].cpu().numpy(), q.cpu().numpy()) < 2e-6
    B.close()


def test_batch3d_rejects_bad_input(astra):
    ang = np.linspace(0, np.pi, 4, endpoint=False).astype(np.float32)
    pg = astra.create_proj_geom('parallel3d', 1.0, 1.0, 4, 4, ang)
    vg = astra.create_vol_geom(4, 4, 4)
    with pytest.raises(astra.AstraError):
        astra.Batch3D([])
    with pytest.raises(astra.AstraError):
        astra.Batch3D([(pg, vg, {'DetectorSuperSampling': 0})])
    B = astra.Batch3D([(pg, vg)])
    with pytest.raises(astra.AstraError):
        B.fp(torch.zeros(3, device='cuda'))
    with pytest.raises(astra.AstraError):
        B.fp(B.empty_vols(), mode=7)
    B.close()
