"""GPU parity of the 3D projectors (b2t_fp3d / b2t_bp3d) against the FP64 oracle.

Tolerances: FP32 storage within 1e-5 relative L2 of the FP64 oracle of the
same ray/voxel model; FP16 / BF16 storage within 1e-3 / 8e-3 of the oracle
evaluated on the rounded input (the output rounding of the storage type).
"""
import ctypes

import numpy as np
import pytest

from conftest import rel_l2

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

TOL_F32 = 1e-5


def _cone_geoms(astra):
    ang = np.linspace(0, 2 * np.pi, 24, endpoint=False).astype(np.float32)
    return [
        ("cone", astra.create_vol_geom(36, 40, 32),
         astra.create_proj_geom('cone', 1.0, 1.0, 40, 48, ang, 150.0, 80.0)),
        ("cone_aniso_window", astra.create_vol_geom(30, 34, 26, -16.0, 18.0, -14.0, 16.0, -12.0, 14.0),
         astra.create_proj_geom('cone', 1.3, 0.8, 36, 44, ang + 0.3, 120.0, 60.0)),
        ("parallel3d", astra.create_vol_geom(36, 40, 32),
         astra.create_proj_geom('parallel3d', 1.0, 1.0, 40, 48, ang[:12] / 2)),
        ("parallel3d_wide", astra.create_vol_geom(28, 30, 20),
         astra.create_proj_geom('parallel3d', 0.7, 1.3, 30, 50, ang[:15])),
    ]


def _vec_geoms(astra):
    rng = np.random.default_rng(5)
    n = 9
    vecs = []
    for i in range(n):
        # source mostly along z for a third of the views (z-major marching)
        t = 2 * np.pi * i / n
        if i % 3 == 0:
            src = np.array([5 * np.cos(t), 5 * np.sin(t), -140.0])
            det = np.array([0.0, 0.0, 70.0])
            u = np.array([np.cos(t), np.sin(t), 0.0])
            v = np.array([-np.sin(t), np.cos(t), 0.0])
        else:
            src = np.array([-140 * np.sin(t), 140 * np.cos(t), 3.0])
            det = np.array([70 * np.sin(t), -70 * np.cos(t), -2.0])
            u = np.array([np.cos(t), np.sin(t), 0.02])
            v = np.array([0.01, 0.0, 1.0])
        u += rng.normal(0, 0.01, 3)
        vecs.append(np.concatenate([src, det, u, v]))
    V = np.array(vecs)
    P = V.copy()
    P[:, 0:3] = P[:, 3:6] - P[:, 0:3]  # parallel: ray direction = detector - source
    P[:, 0:3] /= np.linalg.norm(P[:, 0:3], axis=1, keepdims=True)
    return [
        ("cone_vec", astra.create_vol_geom(34, 30, 28), astra.create_proj_geom('cone_vec', 38, 42, V)),
        ("parallel3d_vec", astra.create_vol_geom(34, 30, 28),
         astra.create_proj_geom('parallel3d_vec', 38, 42, P)),
    ]


def _all_geoms(astra):
    return _cone_geoms(astra) + _vec_geoms(astra)


def _phantom(shape, seed=0):
    rng = np.random.default_rng(seed)
    v = rng.random(shape, dtype=np.float32)
    # smooth-ish content plus an edge so interpolation matters
    v[:, :, : shape[2] // 3] += 1.0
    return v.astype(np.float32)


def _proj(astra, vg, pg, opts=None):
    from importlib import import_module
    P = import_module("astra-toolbox_b200.projector")
    return P.Projector3D(pg, vg, opts or {})


def _oracle_kind(pr):
    return 2 if pr.geom.kind == 2 else 1


@pytest.mark.parametrize("idx", range(6))
def test_fp3d_vs_oracle(astra, orc, idx):
    name, vg, pg = _all_geoms(astra)[idx]
    pr = _proj(astra, vg, pg)
    vol = _phantom(pr.vol_shape, idx)
    tv = torch.from_numpy(vol).cuda()
    tp = torch.full(pr.proj_shape, 7.0, device='cuda')
    pr.fp(tv, tp)
    got = tp.cpu().numpy()
    nv, na, nu = pr.proj_shape
    ref = orc.fp3d(_oracle_kind(pr), pr.geom.views_array(), vol, nu, nv, pr.geom.vol_scale)
    assert rel_l2(got, ref) < TOL_F32, name


@pytest.mark.parametrize("idx", range(6))
def test_bp3d_vs_oracle(astra, orc, idx):
    name, vg, pg = _all_geoms(astra)[idx]
    pr = _proj(astra, vg, pg)
    rng = np.random.default_rng(idx + 10)
    proj = rng.random(pr.proj_shape, dtype=np.float32)
    tp = torch.from_numpy(proj).cuda()
    tv = torch.full(pr.vol_shape, -3.0, device='cuda')
    pr.bp(tp, tv)
    got = tv.cpu().numpy()
    ref = orc.bp3d(_oracle_kind(pr), pr.geom.views_array(), proj, pr.vol_shape, pr.geom.vol_scale)
    assert rel_l2(got, ref) < TOL_F32, name


def test_fp_bp_add_mode(astra):
    name, vg, pg = _cone_geoms(astra)[0]
    pr = _proj(astra, vg, pg)
    vol = torch.from_numpy(_phantom(pr.vol_shape)).cuda()
    p1 = torch.zeros(pr.proj_shape, device='cuda')
    pr.fp(vol, p1)
    p2 = torch.ones(pr.proj_shape, device='cuda')
    pr.fp(vol, p2, mode=0)
    assert torch.allclose(p2, p1 + 1.0, rtol=1e-6, atol=1e-5)
    v1 = torch.zeros(pr.vol_shape, device='cuda')
    pr.bp(p1, v1)
    v2 = torch.full(pr.vol_shape, 2.0, device='cuda')
    pr.bp(p1, v2, mode=0)
    assert torch.allclose(v2, v1 + 2.0, rtol=1e-6, atol=1e-4)


@pytest.mark.parametrize("kind", ["cone", "parallel3d"])
def test_supersampling(astra, orc, kind):
    geoms = {g[0]: g for g in _cone_geoms(astra)}
    _, vg, pg = geoms[kind]
    pr = _proj(astra, vg, pg, {'DetectorSuperSampling': 2, 'VoxelSuperSampling': 2})
    vol = _phantom(pr.vol_shape, 3)
    nv, na, nu = pr.proj_shape
    tp = torch.zeros(pr.proj_shape, device='cuda')
    pr.fp(torch.from_numpy(vol).cuda(), tp)
    ref = orc.fp3d(_oracle_kind(pr), pr.geom.views_array(), vol, nu, nv, pr.geom.vol_scale, rays=2)
    assert rel_l2(tp.cpu().numpy(), ref) < TOL_F32
    proj = np.random.default_rng(4).random(pr.proj_shape, dtype=np.float32)
    tv = torch.zeros(pr.vol_shape, device='cuda')
    pr.bp(torch.from_numpy(proj).cuda(), tv)
    refb = orc.bp3d(_oracle_kind(pr), pr.geom.views_array(), proj, pr.vol_shape, pr.geom.vol_scale, rays=2)
    assert rel_l2(tv.cpu().numpy(), refb) < TOL_F32


@pytest.mark.parametrize("kernel,okernel", [("2d_weighting", 3), ("fdk_weighting", 2)])
def test_bp_weight_kernels(astra, orc, kernel, okernel):
    _, vg, pg = _cone_geoms(astra)[0]
    pr = _proj(astra, vg, pg, {'ProjectionKernel': kernel})
    proj = np.random.default_rng(8).random(pr.proj_shape, dtype=np.float32)
    tv = torch.zeros(pr.vol_shape, device='cuda')
    pr.bp(torch.from_numpy(proj).cuda(), tv)
    ref = orc.bp3d(2, pr.geom.views_array(), proj, pr.vol_shape, pr.geom.vol_scale, kernel=okernel)
    assert rel_l2(tv.cpu().numpy(), ref) < TOL_F32


@pytest.mark.parametrize("idx", [0, 2, 4, 5])
def test_matched_bp_is_exact_transpose(astra, orc, idx):
    name, vg, pg = _all_geoms(astra)[idx]
    pr = _proj(astra, vg, pg, {'ProjectionKernel': 'matched_bp'})
    rng = np.random.default_rng(idx)
    proj = rng.standard_normal(pr.proj_shape).astype(np.float32)
    tv = torch.zeros(pr.vol_shape, device='cuda')
    pr.bp(torch.from_numpy(proj).cuda(), tv)
    ref = orc.fp3d_transpose(_oracle_kind(pr), pr.geom.views_array(), proj, pr.vol_shape, pr.geom.vol_scale)
    assert rel_l2(tv.cpu().numpy(), ref) < TOL_F32, name
    # dot-product test <A x, y> = <x, A^T y> in FP64 accumulation
    x = rng.standard_normal(pr.vol_shape).astype(np.float32)
    ax = torch.zeros(pr.proj_shape, device='cuda')
    pr.fp(torch.from_numpy(x).cuda(), ax)
    lhs = float(np.dot(ax.cpu().numpy().ravel().astype(np.float64), proj.ravel().astype(np.float64)))
    rhs = float(np.dot(x.ravel().astype(np.float64), tv.cpu().numpy().ravel().astype(np.float64)))
    assert abs(lhs - rhs) / abs(lhs) < 1e-5, (lhs, rhs)


@pytest.mark.parametrize("path", ["merged", "plain", "slab"])
def test_matched_bp_fine_detector(astra, orc, path, monkeypatch):
    """Matched BP with a detector finer than the voxels (pixel 0.25 at
    magnification ~2: about four rays per cell along a detector column), so
    runs of three or more lanes fall on one cell in the merged reductions;
    B2T_MATCHED_PLAIN=1 forces the per-lane reductions of very large
    arrays, B2T_MATCHED_PATH=slab the slab transpose (lanes of one shared-
    memory reduction on one cell).  Against the oracle's transpose and the
    dot-product test."""
    if path == "plain":
        monkeypatch.setenv("B2T_MATCHED_PLAIN", "1")
    if path == "slab":
        monkeypatch.setenv("B2T_MATCHED_PATH", "slab")
    ang = np.linspace(0, 2 * np.pi, 12, endpoint=False).astype(np.float32)
    vg = astra.create_vol_geom(24, 28, 20)
    pg = astra.create_proj_geom('cone', 0.25, 0.25, 160, 180, ang, 60.0, 60.0)
    pr = _proj(astra, vg, pg, {'ProjectionKernel': 'matched_bp'})
    rng = np.random.default_rng(21)
    proj = rng.standard_normal(pr.proj_shape).astype(np.float32)
    tv = torch.zeros(pr.vol_shape, device='cuda')
    pr.bp(torch.from_numpy(proj).cuda(), tv)
    ref = orc.fp3d_transpose(2, pr.geom.views_array(), proj, pr.vol_shape, pr.geom.vol_scale)
    assert rel_l2(tv.cpu().numpy(), ref) < TOL_F32
    x = rng.standard_normal(pr.vol_shape).astype(np.float32)
    ax = torch.zeros(pr.proj_shape, device='cuda')
    pr.fp(torch.from_numpy(x).cuda(), ax)
    lhs = float(np.dot(ax.cpu().numpy().ravel().astype(np.float64), proj.ravel().astype(np.float64)))
    rhs = float(np.dot(x.ravel().astype(np.float64), tv.cpu().numpy().ravel().astype(np.float64)))
    assert abs(lhs - rhs) / abs(lhs) < 1e-5, (lhs, rhs)


@pytest.mark.parametrize("dtype,tol", [("float16", 1e-3), ("bfloat16", 8e-3)])
def test_half_storage(astra, orc, dtype, tol):
    _, vg, pg = _cone_geoms(astra)[0]
    pr = _proj(astra, vg, pg)
    tdt = getattr(torch, dtype)
    vol = torch.from_numpy(_phantom(pr.vol_shape, 9)).cuda().to(tdt)
    tp = torch.zeros(pr.proj_shape, device='cuda', dtype=tdt)
    pr.fp(vol, tp)
    nv, na, nu = pr.proj_shape
    ref = orc.fp3d(2, pr.geom.views_array(), vol.float().cpu().numpy(), nu, nv, pr.geom.vol_scale)
    assert rel_l2(tp.float().cpu().numpy(), ref) < tol
    tv = torch.zeros(pr.vol_shape, device='cuda', dtype=tdt)
    pr.bp(tp, tv)
    refb = orc.bp3d(2, pr.geom.views_array(), tp.float().cpu().numpy(), pr.vol_shape, pr.geom.vol_scale)
    assert rel_l2(tv.float().cpu().numpy(), refb) < tol


def test_edge_single_view_single_slice(astra, orc):
    vg = astra.create_vol_geom(17, 23, 1)
    pg = astra.create_proj_geom('cone', 1.0, 1.0, 1, 31, np.array([0.7], dtype=np.float32), 90.0, 40.0)
    pr = _proj(astra, vg, pg)
    vol = _phantom(pr.vol_shape, 2)
    tp = torch.zeros(pr.proj_shape, device='cuda')
    pr.fp(torch.from_numpy(vol).cuda(), tp)
    ref = orc.fp3d(2, pr.geom.views_array(), vol, 31, 1, pr.geom.vol_scale)
    assert rel_l2(tp.cpu().numpy(), ref) < TOL_F32
    tv = torch.zeros(pr.vol_shape, device='cuda')
    pr.bp(tp, tv)
    refb = orc.bp3d(2, pr.geom.views_array(), tp.cpu().numpy(), pr.vol_shape, pr.geom.vol_scale)
    assert rel_l2(tv.cpu().numpy(), refb) < TOL_F32


def test_edge_detector_misses_volume(astra):
    # detector shifted far away: every ray misses, every voxel projects off the detector
    V = np.array([[0, -100, 0, 0, 50, 500, 1, 0, 0, 0, 0, 1]], dtype=np.float64)
    vg = astra.create_vol_geom(16, 16, 16)
    pg = astra.create_proj_geom('cone_vec', 8, 8, V)
    pr = _proj(astra, vg, pg)
    tp = torch.full(pr.proj_shape, 5.0, device='cuda')
    pr.fp(torch.ones(pr.vol_shape, device='cuda'), tp)
    assert float(tp.abs().max()) == 0.0
    tv = torch.full(pr.vol_shape, 5.0, device='cuda')
    pr.bp(torch.ones(pr.proj_shape, device='cuda'), tv)
    assert float(tv.abs().max()) == 0.0


def test_many_views_multiple_launches(astra, orc):
    # more views than one parameter block holds (448 FP / 640 BP per launch)
    ang = np.linspace(0, np.pi, 700, endpoint=False).astype(np.float32)
    vg = astra.create_vol_geom(12, 14, 10)
    pg = astra.create_proj_geom('cone', 1.0, 1.0, 12, 16, ang, 60.0, 30.0)
    pr = _proj(astra, vg, pg)
    vol = _phantom(pr.vol_shape, 1)
    tp = torch.zeros(pr.proj_shape, device='cuda')
    pr.fp(torch.from_numpy(vol).cuda(), tp)
    ref = orc.fp3d(2, pr.geom.views_array(), vol, 16, 12, pr.geom.vol_scale)
    assert rel_l2(tp.cpu().numpy(), ref) < TOL_F32
    proj = tp.cpu().numpy()
    tv = torch.zeros(pr.vol_shape, device='cuda')
    pr.bp(tp, tv)
    refb = orc.bp3d(2, pr.geom.views_array(), proj, pr.vol_shape, pr.geom.vol_scale)
    assert rel_l2(tv.cpu().numpy(), refb) < TOL_F32


def test_errors_are_raised_not_fallen_back(astra):
    _, vg, pg = _cone_geoms(astra)[0]
    pr = _proj(astra, vg, pg)
    with pytest.raises(astra.AstraError):
        pr.fp(torch.zeros(3, 3, 3, device='cuda'), torch.zeros(pr.proj_shape, device='cuda'))
    with pytest.raises(astra.AstraError):
        _proj(astra, vg, pg, {'DetectorSuperSampling': 0}).fp(
            torch.zeros(pr.vol_shape, device='cuda'), torch.zeros(pr.proj_shape, device='cuda'))


def _device_errors():
    import ctypes
    L = __import__("importlib").import_module("astra-toolbox_b200._lib")
    v = ctypes.c_uint32(0)
    L.call("b2t_device_errors", ctypes.byref(v))
    return v.value


def _bp_path_stats():
    L = __import__("importlib").import_module("astra-toolbox_b200._lib")
    st = (ctypes.c_uint64 * 4)()
    L.call("b2t_bp_path_stats", st)
    return list(st)


def _bp_vpt(nz):
    """Voxels per thread of the TMA BP when nothing is tuned: 16 when 1.1 x
    the slices 16-voxel columns compute is fewer than 32-voxel columns do."""
    z16, z32 = 16 * ((nz + 15) // 16), 32 * ((nz + 31) // 32)
    return 16 if 1.1 * z16 < z32 else 32


@pytest.mark.parametrize("dtype", ["float32", "float16", "bfloat16"])
@pytest.mark.parametrize("geom", ["c2_like", "high_mag", "cone_vec", "par3d"])
def test_tma_bp_matches_direct_bp(astra, geom, dtype, monkeypatch):
    """The TMA-staged BP (default) and the direct-load BP implement the same
    model; includes a high-magnification case whose tiles overflow the stage
    (fallback path) and a non-circular cone_vec case.  16-bit projections
    reach the TMA path in the pair layout (two texels per 32-bit word) and the
    direct path as texels."""
    if geom == "c2_like":
        ang = np.linspace(0, 2 * np.pi, 90, endpoint=False).astype(np.float32)
        vg = astra.create_vol_geom(96, 96, 80)
        pg = astra.create_proj_geom('cone', 1.0, 1.0, 100, 110, ang, 190.0, 95.0)
    elif geom == "high_mag":
        ang = np.linspace(0, 2 * np.pi, 30, endpoint=False).astype(np.float32)
        vg = astra.create_vol_geom(64, 64, 40)
        pg = astra.create_proj_geom('cone', 0.25, 0.25, 300, 320, ang, 60.0, 120.0)
    elif geom == "cone_vec":
        _, vg, pg = _vec_geoms(astra)[0]
    else:
        ang = np.linspace(0, np.pi, 50, endpoint=False).astype(np.float32)
        vg = astra.create_vol_geom(70, 60, 50)
        pg = astra.create_proj_geom('parallel3d', 1.0, 1.0, 60, 80, ang)
    pr = _proj(astra, vg, pg)
    tdt = getattr(torch, dtype)
    proj = torch.from_numpy(np.random.default_rng(11).random(pr.proj_shape, dtype=np.float32)).cuda().to(tdt)
    a = torch.zeros(pr.vol_shape, device='cuda', dtype=tdt)
    _bp_path_stats()
    pr.bp(proj, a)
    assert _device_errors() == 0
    fast, general, idle, cycles = _bp_path_stats()
    nz, ny, nx = pr.vol_shape
    # every voxel column (16 or 32 slices per thread) is counted once per
    # view; idle lanes pad the 32 x 8 column blocks
    nviews = pr.proj_shape[1]
    zb = (nz + _bp_vpt(nz) - 1) // _bp_vpt(nz)
    assert fast + general == nx * ny * zb * nviews
    assert idle == (((nx + 31) // 32) * 32 * ((ny + 7) // 8) * 8 - nx * ny) * zb * nviews
    assert cycles > 0
    if geom in ("c2_like", "par3d"):
        assert general == 0
    elif geom == "high_mag":
        assert general > 0
    else:
        assert fast == 0  # non-circular orbit: general path only
    monkeypatch.setenv("B2T_SIMPLE_BP", "1")
    b = torch.zeros(pr.vol_shape, device='cuda', dtype=tdt)
    pr.bp(proj, b)
    monkeypatch.delenv("B2T_SIMPLE_BP")
    # the TMA path takes v at voxel j of a 32-voxel column as v0 + j dv from
    # per-block folded coefficients (rounded to FP32 once); the direct path
    # projects every voxel from the view's coefficients
    # (16-bit: the TMA path interpolates along u in 16-bit arithmetic, and
    # the outputs round to 16 bits)
    tol = {"float32": 4e-6, "float16": 5e-4, "bfloat16": 4e-3}[dtype]
    assert rel_l2(a.float().cpu().numpy(), b.float().cpu().numpy()) < tol


@pytest.mark.parametrize("idx", range(6))
@pytest.mark.parametrize("dtype", ["float32", "float16", "bfloat16"])
def test_cell_fp_matches_padded_fp(astra, idx, dtype, monkeypatch):
    """The cell forward projector (default) and the padded-copy one implement
    the same model, in every storage type and geometry (incl. z-major views)."""
    name, vg, pg = _all_geoms(astra)[idx]
    pr = _proj(astra, vg, pg)
    tdt = getattr(torch, dtype)
    vol = torch.from_numpy(_phantom(pr.vol_shape, idx + 20)).cuda().to(tdt)
    a = torch.zeros(pr.proj_shape, device='cuda', dtype=tdt)
    pr.fp(vol, a)
    monkeypatch.setenv("B2T_SIMPLE_FP", "1")
    b = torch.zeros(pr.proj_shape, device='cuda', dtype=tdt)
    pr.fp(vol, b)
    monkeypatch.delenv("B2T_SIMPLE_FP")
    tol = {"float32": 2e-6, "float16": 2e-3, "bfloat16": 1e-2}[dtype]
    assert rel_l2(a.float().cpu().numpy(), b.float().cpu().numpy()) < tol, name


def _fp_stats():
    import importlib
    L = importlib.import_module("astra-toolbox_b200._lib")
    out = (ctypes.c_uint64 * 4)()
    assert L.load().b2t_fp_path_stats(out) == 0
    return list(out)


def _slab_cases(astra):
    ang = np.linspace(0, 2 * np.pi, 30, endpoint=False).astype(np.float32)
    near45 = np.linspace(np.pi / 4 - 0.2, np.pi / 4 + 0.2, 21).astype(np.float32)
    return {
        # staged slices, rays leaving through every face (clamped slices)
        "cone": (astra.create_vol_geom(40, 44, 36), astra.create_proj_geom('cone', 1.0, 1.0, 48, 56, ang, 150.0, 80.0)),
        "parallel3d": (astra.create_vol_geom(36, 40, 32),
                       astra.create_proj_geom('parallel3d', 1.0, 1.0, 40, 48, ang[:24] / 2)),
        # oblique views: x- and y-major views around 45 degrees, edge rays
        # far outside the volume
        "oblique": (astra.create_vol_geom(48, 40, 30), astra.create_proj_geom('cone', 1.0, 1.0, 40, 96, near45, 90.0, 60.0)),
        # boxes larger than a slice buffer: read from global memory
        "high_mag": (astra.create_vol_geom(40, 40, 40), astra.create_proj_geom('cone', 4.0, 4.0, 36, 20, ang, 60.0, 60.0)),
        # more views than one launch takes, a detector taller than one CTA
        "many_views": (astra.create_vol_geom(20, 18, 24),
                       astra.create_proj_geom('cone', 1.0, 1.0, 150, 22, np.linspace(0, 2 * np.pi, 500, False).astype(np.float32), 80.0, 40.0)),
        # odd sizes, anisotropic voxels
        "odd": (astra.create_vol_geom(17, 23, 9, -9.0, 8.0, -11.0, 12.0, -3.0, 3.0),
                astra.create_proj_geom('cone', 0.7, 1.3, 13, 21, ang + 0.1, 70.0, 30.0)),
        # a detector taller than two CTAs' rows: full row blocks and a partial one
        "tall": (astra.create_vol_geom(32, 36, 60), astra.create_proj_geom('cone', 1.0, 0.4, 44, 340, ang, 150.0, 80.0)),
    }


@pytest.mark.parametrize("case", ["cone", "parallel3d", "oblique", "high_mag", "many_views", "odd", "tall"])
def test_slab_fp_vs_oracle_and_cells(astra, orc, case, monkeypatch):
    """The TMA-staged slab FP (the default for x- and y-major views of
    circular orbits) against the FP64 oracle and against the cell kernels:
    slices staged in shared memory, slices where rays leave the volume
    (clamped to the zero border), slices whose box is too large for a buffer
    (read from global memory), ADD mode, more than one launch of views."""
    vg, pg = _slab_cases(astra)[case]
    pr = _proj(astra, vg, pg)
    vol = _phantom(pr.vol_shape, 31)
    tv = torch.from_numpy(vol).cuda()
    _fp_stats()
    a = torch.zeros(pr.proj_shape, device='cuda')
    pr.fp(tv, a)
    staged, glob, slab_launches, cell_launches = _fp_stats()
    assert slab_launches >= 1 and cell_launches == 0, (case, slab_launches, cell_launches)
    if case == "high_mag":
        assert glob > 0
    else:
        assert staged > 0, (staged, glob)
    nv, na, nu = pr.proj_shape
    ref = orc.fp3d(pr.geom.kind, pr.geom.views_array(), vol, nu, nv, pr.geom.vol_scale)
    assert rel_l2(a.cpu().numpy(), ref) < TOL_F32, case
    monkeypatch.setenv("B2T_FP_PATH", "cells")
    b = torch.zeros(pr.proj_shape, device='cuda')
    pr.fp(tv, b)
    assert _fp_stats()[2] == 0
    monkeypatch.delenv("B2T_FP_PATH")
    assert rel_l2(a.cpu().numpy(), b.cpu().numpy()) < 2e-6, case
    # ADD mode accumulates onto what is there
    c = b.clone()
    pr.fp(tv, c, mode=0)
    assert rel_l2(c.cpu().numpy(), 2 * b.cpu().numpy()) < 2e-6
    flags = ctypes.c_uint32(1)
    import importlib
    assert importlib.import_module("astra-toolbox_b200._lib").load().b2t_device_errors(ctypes.byref(flags)) == 0
    assert flags.value == 0


def _mt_stats():
    import importlib
    L = importlib.import_module("astra-toolbox_b200._lib")
    out = (ctypes.c_uint64 * 4)()
    assert L.load().b2t_matched_path_stats(out) == 0
    return list(out)


@pytest.mark.parametrize("case", ["cone", "parallel3d", "oblique", "high_mag", "many_views", "odd", "tall"])
def test_slab_matched_bp_vs_oracle_and_scatter(astra, orc, case, monkeypatch):
    """The slab FP's transpose (B2T_MATCHED_PATH=slab: shared-memory boxes
    per slice, TMA reduce-adds into the accumulator) against the FP64
    oracle's transpose, against the default per-sample scatter kernels and
    by the dot-product test with the slab FP; boxes too large for a buffer
    scatter straight into global memory (high_mag); ADD mode."""
    vg, pg = _slab_cases(astra)[case]
    pr = _proj(astra, vg, pg, {'ProjectionKernel': 'matched_bp'})
    rng = np.random.default_rng(41)
    proj = rng.standard_normal(pr.proj_shape).astype(np.float32)
    tp = torch.from_numpy(proj).cuda()
    _mt_stats()
    b = torch.zeros(pr.vol_shape, device='cuda')
    pr.bp(tp, b)
    assert _mt_stats()[2] == 0
    monkeypatch.setenv("B2T_MATCHED_PATH", "slab")
    a = torch.zeros(pr.vol_shape, device='cuda')
    pr.bp(tp, a)
    staged, glob, slab_launches, scatter_launches = _mt_stats()
    assert slab_launches >= 1 and scatter_launches == 0, (case, slab_launches, scatter_launches)
    if case == "high_mag":
        assert glob > 0
    else:
        assert staged > 0, (staged, glob)
    ref = orc.fp3d_transpose(_oracle_kind(pr), pr.geom.views_array(), proj, pr.vol_shape, pr.geom.vol_scale)
    assert rel_l2(a.cpu().numpy(), ref) < TOL_F32, case
    assert rel_l2(a.cpu().numpy(), b.cpu().numpy()) < 2e-6, case
    x = rng.standard_normal(pr.vol_shape).astype(np.float32)
    ax = torch.zeros(pr.proj_shape, device='cuda')
    _fp_stats()
    pr.fp(torch.from_numpy(x).cuda(), ax)
    assert _fp_stats()[2] >= 1
    axv = ax.cpu().numpy().ravel().astype(np.float64)
    lhs = float(np.dot(axv, proj.ravel().astype(np.float64)))
    rhs = float(np.dot(x.ravel().astype(np.float64), a.cpu().numpy().ravel().astype(np.float64)))
    # relative to ||A x|| ||y|| (the usual scale of an adjoint test): with
    # zero-mean inputs <A x, y> itself can cancel to far below its terms
    scale = float(np.linalg.norm(axv) * np.linalg.norm(proj.ravel().astype(np.float64)))
    assert abs(lhs - rhs) / scale < 1e-6, (lhs, rhs, scale)
    c = a.clone()
    pr.bp(tp, c, mode=0)
    assert rel_l2(c.cpu().numpy(), 2 * a.cpu().numpy()) < 2e-6
    flags = ctypes.c_uint32(1)
    import importlib
    assert importlib.import_module("astra-toolbox_b200._lib").load().b2t_device_errors(ctypes.byref(flags)) == 0
    assert flags.value == 0


@pytest.mark.parametrize("dtype,tol", [("float16", 1e-3), ("bfloat16", 8e-3)])
def test_slab_matched_bp_16bit(astra, dtype, tol, monkeypatch):
    """16-bit projections and volume through the slab transpose
    (B2T_MATCHED_PATH=slab): the same sums as the scatter kernels up to the
    rounding of the 16-bit output."""
    vg, pg = _slab_cases(astra)["cone"]
    pr = _proj(astra, vg, pg, {'ProjectionKernel': 'matched_bp'})
    tdt = getattr(torch, dtype)
    tp = torch.from_numpy(np.random.default_rng(42).random(pr.proj_shape, dtype=np.float32)).cuda().to(tdt)
    b = torch.zeros(pr.vol_shape, device='cuda', dtype=tdt)
    pr.bp(tp, b)
    monkeypatch.setenv("B2T_MATCHED_PATH", "slab")
    _mt_stats()
    a = torch.zeros(pr.vol_shape, device='cuda', dtype=tdt)
    pr.bp(tp, a)
    assert _mt_stats()[2] >= 1
    assert rel_l2(a.float().cpu().numpy(), b.float().cpu().numpy()) < tol


@pytest.mark.parametrize("dtype", ["float32", "float16"])
def test_autotune_bp3d_shapes_agree(astra, orc, dtype, monkeypatch):
    """The BP autotuner times 32 and 16 voxels per thread and keeps the
    fastest; both shapes backproject the same volume (their per-block folded
    coefficients start at different slices: FP32 rounding apart), every
    column is counted once per view, and the 16-voxel shape matches the
    oracle."""
    ang = np.linspace(0, 2 * np.pi, 60, endpoint=False).astype(np.float32)
    vg = astra.create_vol_geom(72, 64, 40)
    pg = astra.create_proj_geom('cone', 1.0, 1.0, 70, 90, ang, 180.0, 90.0)
    pr = _proj(astra, vg, pg)
    tdt = getattr(torch, dtype)
    proj = torch.from_numpy(np.random.default_rng(13).random(pr.proj_shape, dtype=np.float32)).cuda().to(tdt)
    nz, ny, nx = pr.vol_shape
    out = {}
    for vpt in (32, 16):
        monkeypatch.setenv("B2T_BP_VPT", str(vpt))
        v = torch.zeros(pr.vol_shape, device='cuda', dtype=tdt)
        _bp_path_stats()
        pr.bp(proj, v)
        fast, general, idle, _ = _bp_path_stats()
        assert fast + general == nx * ny * ((nz + vpt - 1) // vpt) * pr.proj_shape[1]
        out[vpt] = v.float().cpu().numpy()
    monkeypatch.delenv("B2T_BP_VPT")
    tol = 4e-6 if dtype == "float32" else 5e-4
    assert rel_l2(out[16], out[32]) < tol
    b = torch.zeros(pr.vol_shape, device='cuda', dtype=tdt)
    vpt = pr.autotune_bp(proj, b)
    assert vpt in (16, 32)
    assert rel_l2(b.float().cpu().numpy(), out[vpt]) < tol
    c = torch.zeros(pr.vol_shape, device='cuda', dtype=tdt)
    pr.bp(proj, c)  # runs with the tuned shape
    assert np.array_equal(c.float().cpu().numpy(), out[vpt])
    refb = orc.bp3d(2, pr.geom.views_array(), proj.float().cpu().numpy(), pr.vol_shape, pr.geom.vol_scale)
    assert rel_l2(out[16], refb) < (1e-5 if dtype == "float32" else 1e-3)


@pytest.mark.parametrize("idx", [0, 4])
def test_autotune_fp3d_keeps_results(astra, orc, idx):
    """The autotuner times the views-per-CTA variants and keeps the fastest;
    every variant computes the same projections."""
    name, vg, pg = _all_geoms(astra)[idx]
    pr = _proj(astra, vg, pg)
    vol = torch.from_numpy(_phantom(pr.vol_shape, idx + 40)).cuda()
    a = torch.zeros(pr.proj_shape, device='cuda')
    pr.fp(vol, a)
    b = torch.zeros(pr.proj_shape, device='cuda')
    vpc = pr.autotune(vol, b)
    assert vpc in (1, 2, 4, 8)
    assert rel_l2(b.cpu().numpy(), a.cpu().numpy()) < 1e-6, name
    c = torch.zeros(pr.proj_shape, device='cuda')
    pr.fp(vol, c)  # runs with the tuned shape
    assert rel_l2(c.cpu().numpy(), a.cpu().numpy()) < 1e-6, name
    ref = orc.fp3d(_oracle_kind(pr), pr.geom.views_array(), vol.cpu().numpy(), pr.proj_shape[2], pr.proj_shape[0],
                   pr.geom.vol_scale)
    assert rel_l2(c.cpu().numpy(), ref) < 1e-5, name


def _sumsqw_geoms(astra):
    ang = np.linspace(0, np.pi, 15, endpoint=False).astype(np.float32)
    par = [g for g in _all_geoms(astra) if g[0].startswith("parallel3d")]
    return par + [("parallel3d_aniso", astra.create_vol_geom(30, 34, 26, -16.0, 18.0, -14.0, 16.0, -12.0, 14.0),
                   astra.create_proj_geom('parallel3d', 0.9, 1.1, 36, 44, ang + 0.2))]


@pytest.mark.parametrize("idx", range(4))
def test_sum_square_weights_vs_oracle(astra, orc, idx):
    """ProjectionKernel 'sum_square_weights' (Par3DFP_SumSqW): every parallel
    geometry, incl. vec views marching along z and anisotropic voxels."""
    name, vg, pg = _sumsqw_geoms(astra)[idx]
    pr = _proj(astra, vg, pg, {'ProjectionKernel': 'sum_square_weights'})
    tp = torch.full(pr.proj_shape, 7.0, device='cuda')
    pr.fp(torch.zeros(pr.vol_shape, device='cuda'), tp)
    nv, na, nu = pr.proj_shape
    ref = orc.par3d_sumsqw(pr.geom.views_array(), pr.vol_shape, nu, nv, pr.geom.vol_scale)
    assert rel_l2(tp.cpu().numpy(), ref) < TOL_F32, name


def test_sum_square_weights_add_mode_and_refusals(astra, orc):
    L = __import__("importlib").import_module("astra-toolbox_b200._lib")
    name, vg, pg = _sumsqw_geoms(astra)[0]
    pr = _proj(astra, vg, pg, {'ProjectionKernel': 'sum_square_weights'})
    tp = torch.ones(pr.proj_shape, device='cuda')
    pr.fp(torch.zeros(pr.vol_shape, device='cuda'), tp, mode=L.MODE_ADD)
    nv, na, nu = pr.proj_shape
    ref = orc.par3d_sumsqw(pr.geom.views_array(), pr.vol_shape, nu, nv, pr.geom.vol_scale)
    assert rel_l2(tp.cpu().numpy(), ref + 1.0) < TOL_F32
    # the reference has it for parallel beams only, without supersampling
    _, cvg, cpg = _cone_geoms(astra)[0]
    cone = _proj(astra, cvg, cpg, {'ProjectionKernel': 'sum_square_weights'})
    with pytest.raises(astra.AstraError):
        cone.fp(torch.zeros(cone.vol_shape, device='cuda'), torch.zeros(cone.proj_shape, device='cuda'))
    ss = _proj(astra, vg, pg, {'ProjectionKernel': 'sum_square_weights', 'DetectorSuperSampling': 2})
    with pytest.raises(astra.AstraError):
        ss.fp(torch.zeros(ss.vol_shape, device='cuda'), torch.zeros(ss.proj_shape, device='cuda'))



def _cyl_case(astra):
    mg = __import__("importlib").import_module("make_golden")
    vg = astra.create_vol_geom(34, 30, 28, -15.0, 15.0, -17.0, 17.0, -14.0, 14.0)
    pg = astra.create_proj_geom('cyl_cone_vec', 40, 46, mg.cyl_vectors())
    return vg, pg


@pytest.fixture
def golden_path():
    import os
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))


def test_cyl_fp_bp_vs_oracle(astra, orc, golden_path):
    """cyl_cone_vec FP and voxel-driven BP (anisotropic voxels, views along
    every axis) against the FP64 oracle, 1e-5."""
    vg, pg = _cyl_case(astra)
    pr = _proj(astra, vg, pg)
    views, vs = pr.geom.views_array(), pr.geom.vol_scale
    nv, na, nu = pr.proj_shape
    vol = _phantom(pr.vol_shape, 3)
    tp = torch.full(pr.proj_shape, 5.0, device='cuda')
    pr.fp(torch.from_numpy(vol).cuda(), tp)
    assert rel_l2(tp.cpu().numpy(), orc.cylcone_fp(views, vol, nu, nv, vs)) < TOL_F32
    proj = np.random.default_rng(4).random(pr.proj_shape).astype(np.float32)
    tv = torch.full(pr.vol_shape, 5.0, device='cuda')
    pr.bp(torch.from_numpy(proj).cuda(), tv)
    assert rel_l2(tv.cpu().numpy(), orc.cylcone_bp(views, proj, pr.vol_shape, vs)) < TOL_F32


def test_cyl_matched_bp_is_exact_transpose(astra, orc, golden_path):
    vg, pg = _cyl_case(astra)
    pr = _proj(astra, vg, pg, {'ProjectionKernel': 'matched_bp'})
    views, vs = pr.geom.views_array(), pr.geom.vol_scale
    rng = np.random.default_rng(5)
    x = torch.from_numpy(rng.standard_normal(pr.vol_shape).astype(np.float32)).cuda()
    y = torch.from_numpy(rng.standard_normal(pr.proj_shape).astype(np.float32)).cuda()
    ax = torch.zeros(pr.proj_shape, device='cuda')
    aty = torch.full(pr.vol_shape, 9.0, device='cuda')
    pr.fp(x, ax)
    pr.bp(y, aty)
    lhs = float((ax.double() * y.double()).sum())
    rhs = float((x.double() * aty.double()).sum())
    assert abs(lhs - rhs) < 1e-5 * abs(lhs)
    want = orc.cylcone_fp_transpose(views, y.cpu().numpy().astype(np.float64), pr.vol_shape, vs)
    assert rel_l2(aty.cpu().numpy(), want) < TOL_F32


def test_cyl_sirt3d_and_refusals(astra, orc, golden_path):
    vg, pg = _cyl_case(astra)
    pr = _proj(astra, vg, pg)
    views, vs = pr.geom.views_array(), pr.geom.vol_scale
    nv, na, nu = pr.proj_shape
    A = lambda x: orc.cylcone_fp(views, x.astype(np.float32), nu, nv, vs)
    B = lambda y: orc.cylcone_bp(views, y.astype(np.float32), pr.vol_shape, vs)
    x_true = np.random.default_rng(6).random(pr.vol_shape).astype(np.float32)
    b = A(x_true).astype(np.float32)
    sid = astra.data3d.create('-proj3d', pg, b)
    rid = astra.data3d.create('-vol', vg, 0)
    cfg = astra.astra_dict('SIRT3D_CUDA')
    cfg['ProjectionDataId'] = sid
    cfg['ReconstructionDataId'] = rid
    aid = astra.algorithm.create(cfg)
    astra.algorithm.run(aid, 4)
    got = astra.data3d.get(rid)
    astra.algorithm.delete(aid)
    # SIRT with the oracle's operators
    inv = lambda a: np.where(a > 1e-6, 1.0 / np.where(a > 1e-6, a, 1.0), 0.0)
    R = inv(A(np.ones(pr.vol_shape)))
    C = inv(B(np.ones(pr.proj_shape)))
    x = np.zeros(pr.vol_shape)
    for _ in range(4):
        x = x + C * B(R * (b - A(x)))
    assert rel_l2(got, x) < 1e-5
    with pytest.raises(astra.AstraError):
        P = __import__("importlib").import_module("astra-toolbox_b200.projector")
        P.fdk(pr, torch.zeros(pr.proj_shape, device='cuda'), torch.zeros(pr.vol_shape, device='cuda'))
    ss = _proj(astra, vg, pg, {'DetectorSuperSampling': 2})
    with pytest.raises(astra.AstraError):
        ss.fp(torch.zeros(ss.vol_shape, device='cuda'), torch.zeros(ss.proj_shape, device='cuda'))
    astra.data3d.delete([sid, rid])
