"""GPU parity of the 2D projectors (b2t_fp2d / b2t_bp2d) against the FP64 oracle
(1e-5 relative L2) and the reference's column-sum known answer."""
import importlib

import numpy as np
import pytest

from conftest import rel_l2

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _geoms(astra):
    rng = np.random.default_rng(7)
    ang = np.linspace(0, np.pi, 45, endpoint=False).astype(np.float32)
    angf = np.linspace(0, 2 * np.pi, 40, endpoint=False).astype(np.float32)
    pv = np.zeros((13, 6))
    fv = np.zeros((13, 6))
    for i in range(13):
        t = 2 * np.pi * i / 13 + 0.1
        pv[i] = [np.sin(t), -np.cos(t), 0.3, -0.2, 1.1 * np.cos(t), 1.1 * np.sin(t)]
        fv[i] = [-90 * np.sin(t), 90 * np.cos(t), 45 * np.sin(t), -45 * np.cos(t), 1.3 * np.cos(t), 1.3 * np.sin(t)]
    return [
        ("parallel", astra.create_vol_geom(48, 56), astra.create_proj_geom('parallel', 1.2, 70, ang)),
        ("fanflat", astra.create_vol_geom(48, 56), astra.create_proj_geom('fanflat', 1.5, 90, angf, 120.0, 60.0)),
        ("parallel_vec", astra.create_vol_geom(40, 44, -20.0, 24.0, -18.0, 22.0),
         astra.create_proj_geom('parallel_vec', 64, pv)),
        ("fanflat_vec", astra.create_vol_geom(40, 44), astra.create_proj_geom('fanflat_vec', 80, fv)),
    ]


def _proj(vg, pg, opts=None):
    P = importlib.import_module("astra-toolbox_b200.projector")
    return P.Projector2D(pg, vg, opts or {})


def _fp_oracle(orc, pr, vol, rays=1):
    f = orc.fan_fp if pr.geom.kind == 4 else orc.par_fp
    return f(pr.geom.views_array(), vol, pr.proj_shape[1], pr.geom.output_scale, rays=rays)


def _bp_oracle(orc, pr, sino, rays=1, fbp=False):
    if pr.geom.kind == 4:
        return orc.fan_bp(pr.geom.views_array(), sino, pr.vol_shape, pr.geom.output_scale, rays=rays, fbp=fbp)
    return orc.par_bp(pr.geom.views_array(), sino, pr.vol_shape, pr.geom.output_scale, rays=rays)


@pytest.mark.parametrize("idx", range(4))
@pytest.mark.parametrize("rays", [1, 3])
def test_fp2d_vs_oracle(astra, orc, idx, rays):
    name, vg, pg = _geoms(astra)[idx]
    pr = _proj(vg, pg, {'DetectorSuperSampling': rays})
    vol = np.random.default_rng(idx).random(pr.vol_shape, dtype=np.float32)
    t = torch.zeros(pr.proj_shape, device='cuda')
    pr.fp(torch.from_numpy(vol).cuda(), t)
    assert rel_l2(t.cpu().numpy(), _fp_oracle(orc, pr, vol, rays)) < 1e-5, name


@pytest.mark.parametrize("idx", range(4))
@pytest.mark.parametrize("rays", [1, 2])
def test_bp2d_vs_oracle(astra, orc, idx, rays):
    name, vg, pg = _geoms(astra)[idx]
    pr = _proj(vg, pg, {'PixelSuperSampling': rays})
    sino = np.random.default_rng(idx + 5).random(pr.proj_shape, dtype=np.float32)
    t = torch.zeros(pr.vol_shape, device='cuda')
    pr.bp(torch.from_numpy(sino).cuda(), t)
    assert rel_l2(t.cpu().numpy(), _bp_oracle(orc, pr, sino, rays)) < 1e-5, name


def test_fan_fbp_weighting(astra, orc):
    name, vg, pg = _geoms(astra)[1]
    pr = _proj(vg, pg)
    sino = np.random.default_rng(3).random(pr.proj_shape, dtype=np.float32)
    t = torch.zeros(pr.vol_shape, device='cuda')
    pr.bp(torch.from_numpy(sino).cuda(), t, fbp_weight=True)
    assert rel_l2(t.cpu().numpy(), _bp_oracle(orc, pr, sino, fbp=True)) < 1e-5


def test_column_sum_known_answer(astra):
    # python/astra/tests.py:28-39 with the 'cuda' projector: 1e-6
    vg = astra.create_vol_geom(2, 32)
    pg = astra.create_proj_geom('parallel', 1, 32, np.array([0.0], dtype=np.float32))
    pr = _proj(vg, pg)
    vol = np.random.default_rng(0).random((2, 32)).astype(np.float32)
    t = torch.zeros(pr.proj_shape, device='cuda')
    pr.fp(torch.from_numpy(vol).cuda(), t)
    assert np.abs(t.cpu().numpy()[0] - vol.sum(axis=0)).max() < 1e-6


def test_add_mode_and_many_views(astra, orc):
    ang = np.linspace(0, 2 * np.pi, 1500, endpoint=False).astype(np.float32)
    vg = astra.create_vol_geom(20, 24)
    pg = astra.create_proj_geom('fanflat', 1.0, 30, ang, 50.0, 25.0)
    pr = _proj(vg, pg)
    vol = np.random.default_rng(1).random(pr.vol_shape, dtype=np.float32)
    t = torch.ones(pr.proj_shape, device='cuda')
    pr.fp(torch.from_numpy(vol).cuda(), t, mode=0)
    assert rel_l2(t.cpu().numpy() - 1.0, _fp_oracle(orc, pr, vol)) < 1e-5
    sino = np.random.default_rng(2).random(pr.proj_shape, dtype=np.float32)
    tv = torch.full(pr.vol_shape, 2.0, device='cuda')
    pr.bp(torch.from_numpy(sino).cuda(), tv, mode=0)
    assert rel_l2(tv.cpu().numpy() - 2.0, _bp_oracle(orc, pr, sino)) < 1e-5
