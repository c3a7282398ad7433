"""GPU parity of FDK (b2t_fdk, b2t_fdk_weight_filter) against the FP64 oracle:
pre-weighting, Parker weighting, exact Toeplitz Ram-Lak filter, FDK BP.
Tolerance 1e-5 relative L2 (FP32 storage)."""
import importlib

import numpy as np
import pytest

from conftest import rel_l2

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _setup(astra, short=False, nu=56, na=72):
    P = importlib.import_module("astra-toolbox_b200.projector")
    if short:
        fan = np.arctan(nu * 0.5 / 300.0)
        ang = np.linspace(0, np.pi + 2 * fan, 60).astype(np.float32)
    else:
        ang = np.linspace(0, 2 * np.pi, na, endpoint=False).astype(np.float32)
    vg = astra.create_vol_geom(36, 36, 28)
    pg = astra.create_proj_geom('cone', 1.0, 1.0, 40, nu, ang, 200.0, 100.0)
    return P, P.Projector3D(pg, vg)


@pytest.mark.parametrize("short", [False, True])
def test_weight_filter_vs_oracle(astra, orc, short):
    P, pr = _setup(astra, short)
    proj = np.random.default_rng(1).random(pr.proj_shape, dtype=np.float32)
    t = torch.from_numpy(proj).cuda()
    P.fdk_weight_filter(pr, t, short_scan=short)
    ref = proj.astype(np.float64)
    orc.fdk_weight(ref, pr.geom.views_array(), short_scan=short)
    orc.ramp_filter_rows(ref)
    assert rel_l2(t.cpu().numpy(), ref) < 1e-5


@pytest.mark.parametrize("short", [False, True])
def test_fdk_vs_oracle(astra, orc, short):
    P, pr = _setup(astra, short)
    vol = np.random.default_rng(2).random(pr.vol_shape, dtype=np.float32)
    tp = torch.zeros(pr.proj_shape, device='cuda')
    pr.fp(torch.from_numpy(vol).cuda(), tp)
    keep = tp.clone()
    rec = torch.zeros(pr.vol_shape, device='cuda')
    P.fdk(pr, tp, rec, short_scan=short)
    assert torch.equal(tp, keep), "b2t_fdk must not modify its input"
    ref = orc.fdk(pr.geom.views_array(), tp.cpu().numpy(), pr.vol_shape, pr.geom.vol_scale, short_scan=short)
    assert rel_l2(rec.cpu().numpy(), ref) < 1e-5


@pytest.mark.parametrize("dtype,tol", [("float16", 2e-3), ("bfloat16", 1.5e-2)])
def test_fdk_16bit_storage(astra, orc, dtype, tol):
    """FDK of 16-bit projections: the filtered rows are stored in 16 bits,
    in the pair layout of the TMA backprojector (written into the second
    half of each row, then rewritten in place as pairs).  Against the oracle
    on the same (16-bit rounded) projections, at the storage precision."""
    P, pr = _setup(astra, nu=60)
    vol = np.random.default_rng(5).random(pr.vol_shape, dtype=np.float32)
    tp = torch.zeros(pr.proj_shape, device='cuda')
    pr.fp(torch.from_numpy(vol).cuda(), tp)
    th = tp.to(getattr(torch, dtype))
    rec = torch.zeros(pr.vol_shape, device='cuda', dtype=th.dtype)
    P.fdk(pr, th, rec)
    ref = orc.fdk(pr.geom.views_array(), th.float().cpu().numpy(), pr.vol_shape, pr.geom.vol_scale)
    assert rel_l2(rec.float().cpu().numpy(), ref) < tol


def test_fdk_no_filter_and_unsupported_filter(astra, orc):
    P, pr = _setup(astra)
    proj = np.random.default_rng(3).random(pr.proj_shape, dtype=np.float32)
    t = torch.from_numpy(proj).cuda()
    P.fdk_weight_filter(pr, t, filter_type='none')
    ref = proj.astype(np.float64)
    orc.fdk_weight(ref, pr.geom.views_array())
    assert rel_l2(t.cpu().numpy(), ref) < 1e-6
    with pytest.raises(astra.AstraError):
        P.filter_code('shepp-logan-typo')


def test_fdk_wide_detector_rows(astra, orc):
    # rows longer than one CTA's default batch: exercises the row-count choice
    P, pr = _setup(astra, nu=1500, na=4)
    proj = np.random.default_rng(4).random(pr.proj_shape, dtype=np.float32)
    t = torch.from_numpy(proj).cuda()
    P.fdk_weight_filter(pr, t)
    ref = proj.astype(np.float64)
    orc.fdk_weight(ref, pr.geom.views_array())
    orc.ramp_filter_rows(ref)
    assert rel_l2(t.cpu().numpy(), ref) < 1e-5
