"""Filters beyond Ram-Lak on the GPU: row filtering (b2t_filter_rows), FDK
and 2D FBP with windowed, cut-off and custom filters against the FP64
oracle's exact Toeplitz filtering with the oracle's own taps (which
tests/test_filters.py pins to the reference's genFilter).  Tolerance 1e-5
relative L2."""
import importlib

import numpy as np
import pytest

from conftest import rel_l2

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _P():
    return importlib.import_module("astra-toolbox_b200.projector")


def _rows(nrows, nu, seed):
    rng = np.random.default_rng(seed)
    u = np.arange(nu)
    out = np.zeros((nrows, nu))
    for _ in range(5):
        cen = rng.uniform(0.1 * nu, 0.9 * nu, size=(nrows, 1))
        w = rng.uniform(0.05 * nu, 0.4 * nu, size=(nrows, 1))
        out += rng.uniform(0, 1, size=(nrows, 1)) * 2 * w * np.sqrt(np.clip(1 - ((u - cen) / w) ** 2, 0, None))
    return (out + 0.01 * rng.standard_normal(out.shape)).astype(np.float32)


CASES = [('shepp-logan', 1.0, -1.0), ('hann', 0.8, -1.0), ('hamming', 1.0, -1.0), ('cosine', 0.6, -1.0),
         ('tukey', 1.0, 0.3), ('kaiser', 1.0, 2.0), ('parzen', 1.0, -1.0), ('ram-lak', 0.5, -1.0)]


@pytest.mark.parametrize("name,d,param", CASES)
def test_filter_rows_vs_oracle(astra, orc, name, d, param):
    P = _P()
    L = importlib.import_module("astra-toolbox_b200._lib")
    lib = L.load()
    nrows, nu = 96, 173
    x = _rows(nrows, nu, seed=hash(name) % 1000)
    spec = P.FilterSpec(name, d=d, parameter=param)
    cfg = spec.c()
    buf = torch.from_numpy(x).cuda()
    import ctypes
    st = lib.b2t_filter_rows(buf.data_ptr(), nrows, nu, nu, ctypes.byref(cfg), torch.cuda.current_stream().cuda_stream)
    assert st == 0, lib.b2t_last_error()
    want = orc.toeplitz_filter_rows(x.astype(np.float64), orc.filter_taps(name, nu, d=d, parameter=param))
    assert rel_l2(buf.cpu().numpy(), want) < 1e-5, name


def test_custom_filters_rows_vs_oracle(astra, orc):
    P = _P()
    L = importlib.import_module("astra-toolbox_b200._lib")
    lib = L.load()
    import ctypes
    rng = np.random.default_rng(11)
    nrows, nu = 40, 90  # rows = views for the per-view types
    F = 256 // 2 + 1
    x = _rows(nrows, nu, seed=2)
    customs = {'projection': rng.random(F), 'sinogram': rng.random((nrows, F)),
               'rprojection': rng.standard_normal(15), 'rsinogram': rng.standard_normal((nrows, 7))}
    for name, custom in customs.items():
        spec = P.FilterSpec(name, custom=custom)
        cfg = spec.c()
        buf = torch.from_numpy(x).cuda()
        st = lib.b2t_filter_rows(buf.data_ptr(), nrows, nu, nu, ctypes.byref(cfg),
                                 torch.cuda.current_stream().cuda_stream)
        assert st == 0, lib.b2t_last_error()
        taps = orc.filter_taps(name, nu, nrows, custom=custom.astype(np.float32))
        want = orc.toeplitz_filter_rows(x.astype(np.float64), taps, set_mod=nrows)
        assert rel_l2(buf.cpu().numpy(), want) < 1e-5, name


@pytest.mark.parametrize("name,d", [('hann', 1.0), ('shepp-logan', 0.7)])
def test_fdk_algorithm_with_filter(astra, orc, name, d):
    ph = importlib.import_module("astra-toolbox_b200.phantom")
    ang = np.linspace(0, 2 * np.pi, 60, endpoint=False).astype(np.float32)
    vg = astra.create_vol_geom(40, 40, 24)
    pg = astra.create_proj_geom('cone', 1.0, 1.0, 32, 150, ang, 200.0, 100.0)
    P = _P()
    pr = P.Projector3D(pg, vg)
    vol = ph.ellipsoids(pr.vol_shape, 6, seed=3, axes=(3.0, 15.0), device='cuda')
    proj = torch.zeros(pr.proj_shape, device='cuda')
    pr.fp(vol, proj)
    pid = astra.data3d.create('-proj3d', pg, proj.cpu().numpy())
    rid = astra.data3d.create('-vol', vg, 0)
    cfg = astra.astra_dict('FDK_CUDA')
    cfg['ProjectionDataId'] = pid
    cfg['ReconstructionDataId'] = rid
    cfg['option'] = {'FilterType': name, 'FilterD': d}
    aid = astra.algorithm.create(cfg)
    astra.algorithm.run(aid)
    got = astra.data3d.get(rid)
    taps = orc.filter_taps(name, pr.proj_shape[2], d=d)
    want = orc.fdk(pr.geom.views_array(), proj.cpu().numpy(), pr.vol_shape, pr.geom.vol_scale, taps=taps)
    assert rel_l2(got, want) < 1e-5, name
    astra.algorithm.delete(aid)


def test_fbp2d_with_filter(astra, orc):
    ang = np.linspace(0, np.pi, 90, endpoint=False).astype(np.float32)
    vg = astra.create_vol_geom(64, 64)
    pg = astra.create_proj_geom('parallel', 1.0, 96, ang)
    pr = astra.Projector2D(pg, vg)
    sino = np.random.default_rng(4).random(pr.proj_shape).astype(np.float32)
    sid = astra.data2d.create('-sino', pg, sino)
    rid = astra.data2d.create('-vol', vg, 0)
    cfg = astra.astra_dict('FBP_CUDA')
    cfg['ProjectionDataId'] = sid
    cfg['ReconstructionDataId'] = rid
    cfg['option'] = {'FilterType': 'hamming'}
    aid = astra.algorithm.create(cfg)
    astra.algorithm.run(aid)
    got = astra.data2d.get(rid)
    filt = orc.toeplitz_filter_rows(sino.astype(np.float64), orc.filter_taps('hamming', pr.proj_shape[1]))
    want = orc.par_bp(pr.geom.views_array(), filt.astype(np.float32), pr.vol_shape,
                      pr.geom.output_scale * (np.pi / 2) / pr.proj_shape[0])
    assert rel_l2(got, want) < 1e-5
