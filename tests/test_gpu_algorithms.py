"""SIRT / CGLS / FBP and the astra-style API on the GPU, against compositions
of the FP64 oracle (SIRT and CGLS recurrences of src/CudaSirtAlgorithm3D.cpp
and src/CudaCglsAlgorithm3D.cpp evaluated in numpy on oracle projections)."""
import importlib

import numpy as np
import pytest

from conftest import rel_l2

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _cone_setup(astra):
    ang = np.linspace(0, 2 * np.pi, 30, endpoint=False).astype(np.float32)
    vg = astra.create_vol_geom(24, 28, 20)
    pg = astra.create_proj_geom('cone', 1.0, 1.0, 26, 34, ang, 120.0, 60.0)
    return vg, pg


def _par2d_setup(astra):
    ang = np.linspace(0, np.pi, 60, endpoint=False).astype(np.float32)
    vg = astra.create_vol_geom(40, 44)
    pg = astra.create_proj_geom('parallel', 1.0, 64, ang)
    return vg, pg


def _ops(orc, pr, is3d):
    """FP64 oracle forward / ASTRA BP as numpy functions."""
    if is3d:
        views, vs = pr.geom.views_array(), pr.geom.vol_scale
        nv, na, nu = pr.proj_shape
        kind = 2 if pr.geom.kind == 2 else 1
        A = lambda x: orc.fp3d(kind, views, x.astype(np.float32), nu, nv, vs)
        B = lambda y: orc.bp3d(kind, views, y.astype(np.float32), pr.vol_shape, vs)
    else:
        views, sc = pr.geom.views_array(), pr.geom.output_scale
        A = lambda x: orc.par_fp(views, x.astype(np.float32), pr.proj_shape[1], sc)
        B = lambda y: orc.par_bp(views, y.astype(np.float32), pr.vol_shape, sc)
    return A, B


def _inv(a):
    out = np.zeros_like(a)
    m = a > 1e-6
    out[m] = 1.0 / a[m]
    return out


def _sirt_ref(A, B, b, x, iters, lam=1.0, vmin=None):
    W_line = _inv(A(np.ones_like(x)))
    W_pix = _inv(B(np.ones_like(b))) * lam
    for _ in range(iters):
        x = x + W_pix * B(W_line * (b - A(x)))
        if vmin is not None:
            x = np.maximum(x, vmin)
    return x


def _cgls_ref(A, B, b, x, iters):
    r = b - A(x)
    p = B(r)
    gamma = float(np.sum(p * p))
    for _ in range(iters):
        w = A(p)
        alpha = gamma / float(np.sum(w * w))
        x = x + alpha * p
        r = r - alpha * w
        z = B(r)
        g2 = float(np.sum(z * z))
        p = z + (g2 / gamma) * p
        gamma = g2
    return x


def _run(astra, vg, pg, kind3d, algo, b, iters, options=None, init=None):
    dm = astra.data3d if kind3d else astra.data2d
    sid = dm.create('-sino', pg, b)
    rid = dm.create('-vol', vg, 0 if init is None else init)
    cfg = astra.astra_dict(algo)
    cfg['ProjectionDataId'] = sid
    cfg['ReconstructionDataId'] = rid
    cfg['option'].update(options or {})
    aid = astra.algorithm.create(cfg)
    astra.algorithm.run(aid, iters)
    out = dm.get(rid)
    res = astra.algorithm.get_res_norm(aid)
    astra.algorithm.delete(aid)
    dm.delete([sid, rid])
    return out, res


@pytest.mark.parametrize("use_graph", [False, True])
def test_sirt3d_vs_oracle(astra, orc, use_graph):
    vg, pg = _cone_setup(astra)
    pr = astra.Projector3D(pg, vg)
    A, B = _ops(orc, pr, True)
    x_true = np.random.default_rng(0).random(pr.vol_shape).astype(np.float32)
    b = A(x_true).astype(np.float32)
    got, res = _run(astra, vg, pg, True, 'SIRT3D_CUDA', b, 6, {'UseGraph': use_graph})
    want = _sirt_ref(A, B, b.astype(np.float64), np.zeros(pr.vol_shape), 6)
    assert rel_l2(got, want) < 1e-5
    assert abs(res - np.linalg.norm(b - A(got))) < 1e-4 * np.linalg.norm(b)


def test_sirt3d_min_constraint_and_relaxation(astra, orc):
    vg, pg = _cone_setup(astra)
    pr = astra.Projector3D(pg, vg)
    A, B = _ops(orc, pr, True)
    x_true = np.random.default_rng(1).standard_normal(pr.vol_shape).astype(np.float32)
    b = A(x_true).astype(np.float32)
    got, _ = _run(astra, vg, pg, True, 'SIRT3D_CUDA', b, 4, {'MinConstraint': 0.0, 'Relaxation': 0.7})
    want = _sirt_ref(A, B, b.astype(np.float64), np.zeros(pr.vol_shape), 4, lam=0.7, vmin=0.0)
    assert got.min() == 0.0
    assert rel_l2(got, want) < 1e-5


@pytest.mark.parametrize("use_graph", [False, True])
def test_cgls3d_vs_oracle(astra, orc, use_graph):
    vg, pg = _cone_setup(astra)
    pr = astra.Projector3D(pg, vg)
    A, B = _ops(orc, pr, True)
    x_true = np.random.default_rng(2).random(pr.vol_shape).astype(np.float32)
    b = A(x_true).astype(np.float32)
    got, res = _run(astra, vg, pg, True, 'CGLS3D_CUDA', b, 5, {'UseGraph': use_graph})
    want = _cgls_ref(A, B, b.astype(np.float64), np.zeros(pr.vol_shape), 5)
    assert rel_l2(got, want) < 1e-4


def test_sirt2d_and_cgls2d_vs_oracle(astra, orc):
    vg, pg = _par2d_setup(astra)
    pr = astra.Projector2D(pg, vg)
    A, B = _ops(orc, pr, False)
    x_true = np.random.default_rng(3).random(pr.vol_shape).astype(np.float32)
    b = A(x_true).astype(np.float32)
    got, _ = _run(astra, vg, pg, False, 'SIRT_CUDA', b, 8)
    want = _sirt_ref(A, B, b.astype(np.float64), np.zeros(pr.vol_shape), 8)
    assert rel_l2(got, want) < 1e-5
    got, _ = _run(astra, vg, pg, False, 'CGLS_CUDA', b, 4)
    want = _cgls_ref(A, B, b.astype(np.float64), np.zeros(pr.vol_shape), 4)
    assert rel_l2(got, want) < 1e-4


def test_fbp2d_parallel_vs_oracle(astra, orc):
    vg, pg = _par2d_setup(astra)
    pr = astra.Projector2D(pg, vg)
    sino = np.random.default_rng(4).random(pr.proj_shape).astype(np.float32)
    got, _ = (None, None)
    sid = astra.data2d.create('-sino', pg, sino)
    rid = astra.data2d.create('-vol', vg, 0)
    cfg = astra.astra_dict('FBP_CUDA')
    cfg['ProjectionDataId'] = sid
    cfg['ReconstructionDataId'] = rid
    aid = astra.algorithm.create(cfg)
    astra.algorithm.run(aid)
    got = astra.data2d.get(rid)
    assert np.array_equal(astra.data2d.get(sid), sino)
    filt = orc.ramp_filter_rows(sino.astype(np.float64))
    want = orc.par_bp(pr.geom.views_array(), filt.astype(np.float32), pr.vol_shape,
                      pr.geom.output_scale * (np.pi / 2) / pr.proj_shape[0])
    assert rel_l2(got, want) < 1e-5


def test_direct_fp3d_matches_create_sino3d_gpu(astra):
    # tests/python/integration/test_dlpack3d.py:123-133 pattern
    vg, pg = _cone_setup(astra)
    vol = np.random.default_rng(5).random((20, 24, 28)).astype(np.float32)
    sid, sino = astra.create_sino3d_gpu(vol, pg, vg)
    pid = astra.create_projector('cuda3d', pg, vg)
    tv = torch.from_numpy(vol).cuda()
    tp = torch.zeros(sino.shape, device='cuda')
    astra.experimental.direct_FP3D(pid, tv, tp)
    assert np.allclose(tp.cpu().numpy(), sino)
    # numpy arrays on the direct path, SET then ADD
    hp = np.zeros(sino.shape, dtype=np.float32)
    astra.experimental.direct_FP3D(pid, vol, hp)
    assert np.allclose(hp, sino)
    astra.experimental.direct_FPBP3D(pid, vol, hp, astra.experimental.MODE_ADD, "FP")
    assert np.allclose(hp, 2 * sino, rtol=1e-5)
    vid, back = astra.create_backprojection3d_gpu(sino, pg, vg)
    hv = np.zeros(vol.shape, dtype=np.float32)
    astra.experimental.direct_BP3D(pid, hv, sino)
    assert np.allclose(hv, back)
    astra.data3d.delete([sid, vid])
    astra.projector3d.delete(pid)


def test_linked_arrays_are_updated(astra):
    vg, pg = _cone_setup(astra)
    vol = np.random.default_rng(6).random((20, 24, 28)).astype(np.float32)
    sino = np.zeros((26, 30, 34), dtype=np.float32)
    vid = astra.data3d.link('-vol', vg, vol)
    sid = astra.data3d.link('-sino', pg, sino)
    cfg = astra.astra_dict('FP3D_CUDA')
    cfg['VolumeDataId'] = vid
    cfg['ProjectionDataId'] = sid
    aid = astra.algorithm.create(cfg)
    astra.algorithm.run(aid)
    assert np.abs(sino).max() > 0 and np.array_equal(sino, astra.data3d.get(sid))
    with pytest.raises(astra.AstraError):
        astra.data3d.link('-vol', vg, vol[:, :, ::2])
    astra.algorithm.delete(aid)
    astra.data3d.delete([vid, sid])


def test_fdk_algorithm_object(astra, orc):
    ang = np.linspace(0, 2 * np.pi, 48, endpoint=False).astype(np.float32)
    vg = astra.create_vol_geom(24, 24, 16)
    pg = astra.create_proj_geom('cone', 1.0, 1.0, 20, 36, ang, 150.0, 75.0)
    pr = astra.Projector3D(pg, vg)
    proj = np.random.default_rng(7).random(pr.proj_shape).astype(np.float32)
    sid = astra.data3d.create('-sino', pg, proj)
    rid = astra.data3d.create('-vol', vg, 0)
    cfg = astra.astra_dict('FDK_CUDA')
    cfg['ProjectionDataId'] = sid
    cfg['ReconstructionDataId'] = rid
    aid = astra.algorithm.create(cfg)
    astra.algorithm.run(aid)
    want = orc.fdk(pr.geom.views_array(), proj, pr.vol_shape, pr.geom.vol_scale)
    assert rel_l2(astra.data3d.get(rid), want) < 1e-5
    astra.algorithm.delete(aid)
    astra.data3d.delete([sid, rid])


def test_optomo_matches_projector_and_solves(astra, orc):
    """OpTomo (python/astra/optomo.py interface): W * x, W.T * s on numpy and
    CUDA tensors equal the projector's FP / BP; scipy lsqr runs on it."""
    import scipy.sparse.linalg
    vg, pg = _par2d_setup(astra)
    pid = astra.create_projector('cuda', pg, vg)
    W = astra.OpTomo(pid)
    pr = astra.Projector2D(pg, vg)
    x = np.random.default_rng(8).random(pr.vol_shape).astype(np.float32)
    s = W * x
    ref = torch.zeros(pr.proj_shape, device='cuda')
    pr.fp(torch.from_numpy(x).cuda(), ref)
    assert np.array_equal(s, ref.cpu().numpy())
    b = W.T * s
    refb = torch.zeros(pr.vol_shape, device='cuda')
    pr.bp(ref, refb)
    assert np.array_equal(b, refb.cpu().numpy())
    # flattened vectors and CUDA tensors
    assert np.array_equal(W.matvec(x.ravel()), s.ravel())
    tx = torch.from_numpy(x).cuda()
    assert torch.equal(W * tx, ref)
    assert W.shape == (s.size, x.size)
    sol = scipy.sparse.linalg.lsqr(W, s.ravel(), iter_lim=20)[0]
    assert np.linalg.norm(W.matvec(sol) - s.ravel()) < 0.2 * np.linalg.norm(s)
    rec = W.reconstruct('SIRT_CUDA', s, 20)
    assert rec.shape == pr.vol_shape and np.isfinite(rec).all()


def _fan2d_setup(astra):
    ang = np.linspace(0, 2 * np.pi, 50, endpoint=False).astype(np.float32)
    vg = astra.create_vol_geom(36, 40)
    pg = astra.create_proj_geom('fanflat', 1.2, 70, ang, 110.0, 50.0)
    return vg, pg


@pytest.mark.parametrize("geom", ["parallel", "fanflat"])
def test_sart2d_vs_oracle(astra, orc, geom):
    """SART_CUDA, sequential order, two sweeps, min constraint and relaxation,
    against the oracle's single-view steps (float state in both: 1e-4)."""
    vg, pg = (_par2d_setup if geom == "parallel" else _fan2d_setup)(astra)
    pr = astra.Projector2D(pg, vg)
    kind = pr.geom.kind
    views, sc = pr.geom.views_array(), pr.geom.output_scale
    fp = orc.par_fp if kind == 3 else orc.fan_fp
    x_true = np.random.default_rng(5).random(pr.vol_shape).astype(np.float32)
    b = fp(views, x_true, pr.proj_shape[1], sc).astype(np.float32)
    iters = 2 * pr.proj_shape[0]
    opts = {'ProjectionOrder': 'sequential', 'MinConstraint': 0.0, 'Relaxation': 0.8}
    got, res = _run(astra, vg, pg, False, 'SART_CUDA', b, iters, opts)
    want = orc.sart2d(kind, views, b, np.zeros(pr.vol_shape), sc, iters, lam=0.8, min_value=0.0)
    assert rel_l2(got, want) < 1e-4, rel_l2(got, want)
    assert got.min() >= 0.0
    assert abs(res - np.linalg.norm(b - fp(views, got, pr.proj_shape[1], sc))) < 1e-4 * np.linalg.norm(b)


def test_sart2d_custom_order_runs_resume_and_graph(astra, orc):
    """A custom ProjectionOrderList used cyclically; the step count carries
    over between run() calls; the CUDA-graph replay gives identical results."""
    vg, pg = _par2d_setup(astra)
    pr = astra.Projector2D(pg, vg)
    views, sc = pr.geom.views_array(), pr.geom.output_scale
    x_true = np.random.default_rng(6).random(pr.vol_shape).astype(np.float32)
    b = orc.par_fp(views, x_true, pr.proj_shape[1], sc).astype(np.float32)
    order = np.random.default_rng(7).permutation(pr.proj_shape[0])[:25]
    want = orc.sart2d(3, views, b, np.zeros(pr.vol_shape), sc, 70, order=order)
    outs = []
    for graph in (False, True):
        sid = astra.data2d.create('-sino', pg, b)
        rid = astra.data2d.create('-vol', vg, 0)
        cfg = astra.astra_dict('SART_CUDA')
        cfg['ProjectionDataId'] = sid
        cfg['ReconstructionDataId'] = rid
        cfg['option'] = {'ProjectionOrder': 'custom', 'ProjectionOrderList': order, 'UseGraph': graph}
        aid = astra.algorithm.create(cfg)
        astra.algorithm.run(aid, 30)
        astra.algorithm.run(aid, 40)
        outs.append(astra.data2d.get(rid))
        astra.algorithm.delete(aid)
        astra.data2d.delete([sid, rid])
    assert rel_l2(outs[0], want) < 1e-4
    assert np.array_equal(outs[0], outs[1])


def test_sart2d_mask_and_refusals(astra, orc):
    vg, pg = _fan2d_setup(astra)
    pr = astra.Projector2D(pg, vg)
    views, sc = pr.geom.views_array(), pr.geom.output_scale
    x_true = np.random.default_rng(8).random(pr.vol_shape).astype(np.float32)
    b = orc.fan_fp(views, x_true, pr.proj_shape[1], sc).astype(np.float32)
    mask = np.zeros(pr.vol_shape, dtype=np.float32)
    mask[5:30, 6:34] = 1.0
    mid = astra.data2d.create('-vol', vg, mask)
    got, _ = _run(astra, vg, pg, False, 'SART_CUDA', b, 50,
                  {'ProjectionOrder': 'sequential', 'ReconstructionMaskId': mid})
    want = orc.sart2d(4, views, b, np.zeros(pr.vol_shape), sc, 50, mask=mask)
    assert rel_l2(got, want) < 1e-4
    assert np.all(got[mask == 0] == 0.0)
    sm = astra.data2d.create('-sino', pg, np.ones_like(b))
    with pytest.raises(astra.AstraError):
        _run(astra, vg, pg, False, 'SART_CUDA', b, 1, {'SinogramMaskId': sm})
    with pytest.raises(astra.AstraError):
        _run(astra, vg, pg, False, 'SART_CUDA', b, 1,
             {'ProjectionOrder': 'custom', 'ProjectionOrderList': [0, 1, 999]})
    astra.data2d.delete([mid, sm])
