"""Tensor-core Ram-Lak filter (tcgen05, split BF16 x 6 products, FP32
accumulation) against the FP64 oracle's exact Toeplitz filter, against the
SIMT filter, and inside FDK.  Rows are projection-like (smooth, positive,
strongly cancelling under the ramp filter), the hard case for split-precision
products.  Tolerance: 1e-5 relative L2."""
import ctypes
import importlib
import os

import numpy as np
import pytest

from conftest import rel_l2

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _lib():
    L = importlib.import_module("astra-toolbox_b200._lib")
    return L, L.load()


def _rows(nrows, nu, seed):
    """Line integrals of random ellipses (smooth bumps) plus a little noise."""
    rng = np.random.default_rng(seed)
    u = np.arange(nu, dtype=np.float64)
    out = np.zeros((nrows, nu))
    for _ in range(6):
        cen = rng.uniform(0.1 * nu, 0.9 * nu, size=(nrows, 1))
        w = rng.uniform(0.05 * nu, 0.4 * nu, size=(nrows, 1))
        a = rng.uniform(0.0, 1.0, size=(nrows, 1))
        out += a * 2 * w * np.sqrt(np.clip(1 - ((u - cen) / w) ** 2, 0, None))
    out += 1e-3 * out.max() * rng.standard_normal(out.shape)
    return out.astype(np.float32)


def _filter(x, pitch=None, simt=False):
    L, lib = _lib()
    nrows, nu = x.shape
    pitch = pitch or nu
    buf = torch.zeros((nrows, pitch), dtype=torch.float32, device="cuda")
    buf[:, :nu] = torch.from_numpy(x).cuda()
    old = os.environ.get("B2T_SIMT_FILTER")
    os.environ["B2T_SIMT_FILTER"] = "1" if simt else "0"
    try:
        n0 = lib.b2t_kernel_launches()
        cfg = L.FilterConfig(L.FILTER_RAMLAK, 1.0, -1.0, None, 0, 0)
        st = lib.b2t_filter_rows(buf.data_ptr(), nrows, nu, pitch, ctypes.byref(cfg),
                                 torch.cuda.current_stream().cuda_stream)
        assert st == L.B2T_OK, lib.b2t_last_error()
        torch.cuda.synchronize()
        launches = lib.b2t_kernel_launches() - n0
    finally:
        if old is None:
            del os.environ["B2T_SIMT_FILTER"]
        else:
            os.environ["B2T_SIMT_FILTER"] = old
    flags = ctypes.c_uint32(0)
    assert lib.b2t_device_errors(ctypes.byref(flags)) == L.B2T_OK and flags.value == 0
    return buf[:, :nu].cpu().numpy(), buf[:, nu:].cpu().numpy(), launches


@pytest.mark.parametrize("nrows,nu,pitch", [(128, 127, None), (300, 256, None), (517, 301, 307),
                                            (1024, 832, None), (200, 1500, None)])
def test_tc_filter_vs_oracle(orc, nrows, nu, pitch):
    x = _rows(nrows, nu, seed=nu)
    got, tail, launches = _filter(x, pitch)
    ref = orc.ramp_filter_rows(x.astype(np.float64))
    err = rel_l2(got, ref)
    assert err < 1e-5, err
    assert launches == 3  # split, taps, tcgen05 GEMM
    if tail.size:
        assert not tail.any(), "pitch padding must stay untouched"


def test_tc_filter_not_worse_than_simt(orc):
    x = _rows(640, 832, seed=7)
    ref = orc.ramp_filter_rows(x.astype(np.float64))
    tc, _, n_tc = _filter(x)
    simt, _, n_simt = _filter(x, simt=True)
    assert n_tc == 3 and n_simt == 1
    e_tc, e_simt = rel_l2(tc, ref), rel_l2(simt, ref)
    assert e_tc < 1e-5 and e_tc < 2.0 * e_simt + 1e-7, (e_tc, e_simt)


def test_small_shapes_use_simt(orc):
    # fewer than 127 columns or 128 rows: SIMT kernel (one launch)
    for nrows, nu in ((64, 400), (400, 100)):
        x = _rows(nrows, nu, seed=3)
        got, _, launches = _filter(x)
        assert launches == 1
        assert rel_l2(got, orc.ramp_filter_rows(x.astype(np.float64))) < 1e-5


@pytest.mark.parametrize("short", [False, True])
def test_fdk_with_tc_filter_vs_oracle(astra, orc, short):
    P = importlib.import_module("astra-toolbox_b200.projector")
    ph = importlib.import_module("astra-toolbox_b200.phantom")
    nu, nv = 200, 48
    if short:
        fan = np.arctan(nu * 0.5 / 300.0)
        ang = np.linspace(0, np.pi + 2 * fan, 100).astype(np.float32)
    else:
        ang = np.linspace(0, 2 * np.pi, 90, endpoint=False).astype(np.float32)
    vg = astra.create_vol_geom(64, 64, 40)
    pg = astra.create_proj_geom('cone', 1.0, 1.0, nv, nu, ang, 200.0, 100.0)
    pr = P.Projector3D(pg, vg)
    vol = ph.ellipsoids(pr.vol_shape, 8, seed=5, axes=(4.0, 24.0), device='cuda')
    proj = torch.zeros(pr.proj_shape, device='cuda')
    pr.fp(vol, proj)
    rec = torch.zeros(pr.vol_shape, device='cuda')
    P.fdk(pr, proj, rec, short_scan=short)
    ref = orc.fdk(pr.geom.views_array(), proj.cpu().numpy(), pr.vol_shape, pr.geom.vol_scale, short_scan=short)
    err = rel_l2(rec.cpu().numpy(), ref)
    assert err < 1e-5, err
    # in-place weighting + filtering through the same path
    wf = proj.clone()
    P.fdk_weight_filter(pr, wf, short_scan=short)
    r2 = proj.cpu().numpy().astype(np.float64)
    orc.fdk_weight(r2, pr.geom.views_array(), short_scan=short)
    orc.ramp_filter_rows(r2)
    assert rel_l2(wf.cpu().numpy(), r2) < 1e-5


@pytest.mark.parametrize("dtype,tol", [(torch.float16, 2e-3), (torch.bfloat16, 1e-2)])
def test_fdk_half_storage_tc(astra, orc, dtype, tol):
    P = importlib.import_module("astra-toolbox_b200.projector")
    ph = importlib.import_module("astra-toolbox_b200.phantom")
    ang = np.linspace(0, 2 * np.pi, 90, endpoint=False).astype(np.float32)
    vg = astra.create_vol_geom(64, 64, 40)
    pg = astra.create_proj_geom('cone', 1.0, 1.0, 48, 200, ang, 200.0, 100.0)
    pr = P.Projector3D(pg, vg)
    vol = ph.ellipsoids(pr.vol_shape, 8, seed=6, axes=(4.0, 24.0), device='cuda')
    proj = torch.zeros(pr.proj_shape, device='cuda')
    pr.fp(vol, proj)
    rec = torch.zeros(pr.vol_shape, device='cuda', dtype=dtype)
    P.fdk(pr, proj.to(dtype), rec, short_scan=False)
    ref = orc.fdk(pr.geom.views_array(), proj.to(dtype).float().cpu().numpy(), pr.vol_shape, pr.geom.vol_scale)
    err = rel_l2(rec.float().cpu().numpy(), ref)
    assert err < tol, err
