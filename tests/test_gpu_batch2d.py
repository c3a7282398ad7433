"""Batched 2D problems (b2t_batch2d_*): one persistent launch per operation for
a mixed batch of parallel and fan problems of different sizes, angle counts
and supersampling, against the single-problem projectors (same arithmetic:
FP bit for bit, BP bit for bit up to 1024 views) and batched SIRT against
per-problem SIRT_CUDA."""
import importlib

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _problems(astra, seed=0, big_views=False):
    rng = np.random.default_rng(seed)
    probs = []
    for i in range(9):
        W = int(rng.choice([24, 40, 64, 96]))
        H = W if i % 3 else W + 8
        na = int(rng.integers(12, 90))
        if big_views and i == 0:
            na = 1100
        nd = int(1.5 * W)
        ang = np.linspace(0, 2 * np.pi, na, endpoint=False).astype(np.float32)
        vg = astra.create_vol_geom(H, W)
        if i % 2 == 0:
            pg = astra.create_proj_geom('fanflat', 1.0, nd, ang, 2.0 * W, 1.0 * W)
        else:
            pg = astra.create_proj_geom('parallel', 1.0, nd, ang[: max(2, na // 2)])
        opts = {'DetectorSuperSampling': 2, 'PixelSuperSampling': 2} if i == 4 else {}
        probs.append((pg, vg, opts))
    return probs


def _phantoms(batch, seed=1):
    rng = np.random.default_rng(seed)
    return [torch.from_numpy(rng.random(sh, dtype=np.float32)).cuda() for sh in batch.vol_shapes]


@pytest.mark.parametrize("big_views", [False, True])
def test_batched_fp_bp_match_single_problem(astra, big_views):
    L = importlib.import_module("astra-toolbox_b200._lib")
    lib = L.load()
    probs = _problems(astra, big_views=big_views)
    B = astra.Batch2D(probs)
    vols = B.pack_vols(_phantoms(B))
    n0 = lib.b2t_kernel_launches()
    sinos = B.fp(vols)
    torch.cuda.synchronize()
    assert lib.b2t_kernel_launches() - n0 == 1, "one persistent launch for the whole batch"
    back = B.bp(sinos)
    for i, (pg, vg, opts) in enumerate(probs):
        pr = astra.Projector2D(pg, vg, opts)
        v = B.vol_views(vols)[i].contiguous()
        s1 = torch.zeros(pr.proj_shape, device='cuda')
        pr.fp(v, s1)
        assert torch.equal(B.sino_views(sinos)[i], s1), i
        b1 = torch.zeros(pr.vol_shape, device='cuda')
        pr.bp(B.sino_views(sinos)[i].contiguous(), b1)
        bb = B.vol_views(back)[i]
        if pr.proj_shape[0] <= 1024:
            assert torch.equal(bb, b1), i
        else:
            assert float((bb - b1).norm() / b1.norm()) < 1e-6, i
    # accumulate mode adds
    sinos2 = sinos.clone()
    B.fp(vols, sinos2, mode=L.MODE_ADD)
    assert torch.allclose(sinos2, 2 * sinos, rtol=1e-6, atol=1e-6)
    B.close()


def test_batched_sirt_matches_per_problem(astra):
    A = importlib.import_module("astra-toolbox_b200.algorithm")
    D = importlib.import_module("astra-toolbox_b200.data2d")
    probs = _problems(astra, seed=3)
    B = astra.Batch2D(probs)
    truth = B.pack_vols(_phantoms(B, seed=4))
    sinos = B.fp(truth)
    rec = B.empty_vols()
    res = B.sirt(sinos, rec, 20, min_constraint=0.0)
    assert np.isfinite(res)
    for i, (pg, vg, opts) in enumerate(probs):
        sid = D.create('-sino', pg, B.sino_views(sinos)[i].cpu().numpy())
        vid = D.create('-vol', vg, 0)
        pid = astra.create_projector('cuda', pg, vg, opts)
        cfg = astra.astra_dict('SIRT_CUDA')
        cfg['ProjectorId'] = pid
        cfg['ProjectionDataId'] = sid
        cfg['ReconstructionDataId'] = vid
        cfg['option'] = {'MinConstraint': 0.0}
        aid = A.create(cfg)
        A.run(aid, 20)
        ref = torch.from_numpy(D.get(vid)).cuda()
        got = B.vol_views(rec)[i]
        assert float((got - ref).norm() / ref.norm()) < 1e-6, i
        A.delete(aid)
        D.delete([sid, vid])
    B.close()


def test_batched_cgls_matches_per_problem(astra):
    A = importlib.import_module("astra-toolbox_b200.algorithm")
    D = importlib.import_module("astra-toolbox_b200.data2d")
    probs = _problems(astra, seed=5)
    B = astra.Batch2D(probs)
    truth = B.pack_vols(_phantoms(B, seed=6))
    sinos = B.fp(truth)
    rec = B.empty_vols()
    res = B.cgls(sinos, rec, 10)
    assert np.isfinite(res)
    for i, (pg, vg, opts) in enumerate(probs):
        sid = D.create('-sino', pg, B.sino_views(sinos)[i].cpu().numpy())
        vid = D.create('-vol', vg, 0)
        pid = astra.create_projector('cuda', pg, vg, opts)
        cfg = astra.astra_dict('CGLS_CUDA')
        cfg['ProjectorId'] = pid
        cfg['ProjectionDataId'] = sid
        cfg['ReconstructionDataId'] = vid
        aid = A.create(cfg)
        A.run(aid, 10)
        ref = torch.from_numpy(D.get(vid)).cuda()
        got = B.vol_views(rec)[i]
        # same operator and recurrences; FP64 sums over a different chunking
        assert float((got - ref).norm() / ref.norm()) < 1e-4, i
        A.delete(aid)
        D.delete([sid, vid])
    B.close()


def test_batch_rejects_bad_input(astra):
    with pytest.raises(astra.AstraError):
        astra.Batch2D([])
    probs = _problems(astra)
    B = astra.Batch2D(probs)
    with pytest.raises(astra.AstraError):
        B.fp(torch.zeros(3, device='cuda'))
    B.close()
