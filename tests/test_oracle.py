"""The FP64 oracle against the reference's known answers and its own invariants (CPU)."""
import numpy as np
import pytest

from conftest import rel_l2


def _par3d(astra, geo, shape, angles, det):
    vg = astra.create_vol_geom(*shape)
    pg = astra.create_proj_geom('parallel3d', 1, 1, det[0], det[1], np.asarray(angles, dtype=np.float32))
    return geo.Geometry3D(vg, pg)


def test_par3d_column_sum_known_answer(astra, geo, orc):
    # python/astra/tests.py:41-50: axis-aligned parallel FP equals the column sum (1e-6)
    g = _par3d(astra, geo, (2, 32, 32), [0.0], (32, 32))
    vol = np.random.default_rng(0).random((32, 2, 32)).astype(np.float32)
    p = orc.fp3d(orc.PAR3D, g.views_array(), vol, 32, 32, g.vol_scale)
    assert np.abs(p[:, 0, :] - vol.astype(np.float64).sum(axis=1)).max() < 1e-6


def test_par3d_sum_square_weights_known_answer(astra, geo, orc):
    # axis-aligned rays through voxel centres weigh every crossed voxel by 1 in
    # both plane axes, so each ray's sum is the slice count (2 here); a detector
    # shifted by half a voxel puts every ray on a texel boundary: 0.5^2 + 0.5^2
    # per axis, except the outer rays, which keep one neighbour (0.5^2)
    g = _par3d(astra, geo, (2, 8, 6), [0.0], (6, 8))
    p = orc.par3d_sumsqw(g.views_array(), (6, 2, 8), 8, 6, g.vol_scale)
    assert np.abs(p[:, 0, :] - 2.0).max() < 1e-12
    vg = astra.create_vol_geom(2, 8, 6)
    pg = astra.create_proj_geom('parallel3d_vec', 6, 9, np.array([[0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1]], float))
    g2 = geo.Geometry3D(vg, pg)
    p2 = orc.par3d_sumsqw(g2.views_array(), (6, 2, 8), 9, 6, g2.vol_scale)
    want = np.full(9, 0.5)
    want[[0, 8]] = 0.25
    assert np.abs(p2[:, 0, :] - 2.0 * want[None, :]).max() < 1e-12


def test_par2d_column_sum_known_answer(astra, geo, orc):
    # python/astra/tests.py:28-39 ('cuda' projector): column sums, 1e-6
    vg = astra.create_vol_geom(2, 32)
    pg = astra.create_proj_geom('parallel', 1, 32, np.array([0.0], dtype=np.float32))
    g = geo.Geometry2D(vg, pg)
    vol = np.random.default_rng(1).random((2, 32)).astype(np.float32)
    s = orc.par_fp(g.views_array(), vol, 32, g.output_scale)
    assert np.abs(s[0] - vol.astype(np.float64).sum(axis=0)).max() < 1e-6


@pytest.mark.parametrize("kind", ["cone", "parallel3d"])
def test_fp_transpose_dot_product(astra, geo, orc, kind):
    rng = np.random.default_rng(3)
    vg = astra.create_vol_geom(14, 12, 10)
    ang = np.linspace(0, 2 * np.pi, 7, endpoint=False).astype(np.float32)
    if kind == "cone":
        pg = astra.create_proj_geom('cone', 1.0, 1.0, 12, 16, ang, 50.0, 25.0)
    else:
        pg = astra.create_proj_geom('parallel3d', 1.0, 1.0, 12, 16, ang)
    g = geo.Geometry3D(vg, pg)
    k = orc.CONE if kind == "cone" else orc.PAR3D
    x = rng.standard_normal((10, 12, 14)).astype(np.float32)
    y = rng.standard_normal((12, 7, 16))
    ax = orc.fp3d(k, g.views_array(), x, 16, 12, g.vol_scale)
    aty = orc.fp3d_transpose(k, g.views_array(), y, (10, 12, 14), g.vol_scale)
    lhs = float(np.dot(ax.ravel(), y.ravel()))
    rhs = float(np.dot(x.astype(np.float64).ravel(), aty.ravel()))
    assert abs(lhs - rhs) < 1e-12 * max(1.0, abs(lhs))


def test_ramp_filter_equals_padded_fft_convolution(orc):
    # generateRampFilter (src/Filters.cpp:41-69) on the nextpow2(2n) grid,
    # applied by zero-padded FFT, is the Toeplitz product the oracle evaluates
    n = 37
    N = 1 << int(np.ceil(np.log2(2 * n)))
    h = np.zeros(N)
    for i in range(N):
        if i & 1:
            j = i if 2 * i <= N else N - i
            h[i] = -1.0 / (np.pi * j) ** 2
    h[0] = 0.25
    H = 2.0 * np.fft.fft(h).real
    x = np.random.default_rng(2).standard_normal((5, n))
    xp = np.zeros((5, N))
    xp[:, :n] = x
    ref = np.fft.ifft(np.fft.fft(xp, axis=1) * H[None, :], axis=1).real[:, :n]
    got = orc.ramp_filter_rows(x.copy())
    assert np.abs(got - ref).max() < 1e-12


def test_bp_matches_brute_force_voxel_projection(astra, geo, orc):
    # one view, cone: the BP value of a voxel is the bilinear sample of the
    # projection at the voxel centre's detector coordinates times the weight
    vg = astra.create_vol_geom(6, 5, 4)
    pg = astra.create_proj_geom('cone', 1.0, 1.0, 6, 7, np.array([0.4], dtype=np.float32), 30.0, 20.0)
    g = geo.Geometry3D(vg, pg)
    proj = np.random.default_rng(0).random((6, 1, 7)).astype(np.float32)
    vol = orc.bp3d(orc.CONE, g.views_array(), proj, (4, 5, 6), g.vol_scale)
    w = g.views_array()[0]
    S, D, U, V = w[0:3], w[3:6], w[6:9], w[9:12]
    X, Y, Z = 2, 3, 1
    x = np.array([X - 3 + 0.5, Y - 2.5 + 0.5, Z - 2 + 0.5])
    # intersect the ray S->x with the detector plane D + a U + b V
    M = np.stack([U, V, -(x - S)], axis=1)
    a, b, t = np.linalg.solve(M, S - D)
    qa, qb = a - 0.5, b - 0.5
    ka, kb = int(np.floor(qa)), int(np.floor(qb))
    fa, fb = qa - ka, qb - kb
    P = proj[:, 0, :].astype(np.float64)
    val = ((1 - fa) * (1 - fb) * P[kb, ka] + fa * (1 - fb) * P[kb, ka + 1] + (1 - fa) * fb * P[kb + 1, ka]
           + fa * fb * P[kb + 1, ka + 1])
    uv = np.cross(U, V)
    smd = S - D
    # ray-density weight 1/Den^2 = det(u,v,s-d)^2 / (|u x v| det(u,v,s-x)^2) (cone_bp.cu:226-295)
    wgt = (np.dot(uv, smd) / np.dot(uv, S - x)) ** 2 / np.linalg.norm(uv)
    assert abs(vol[Z, Y, X] - val * wgt) < 1e-9 * max(1.0, abs(val * wgt))


def test_dominant_axis_matches_rule(astra, geo, orc):
    vg = astra.create_vol_geom(8, 8, 8)
    ang = np.array([0.0, np.pi / 2, np.pi / 4, 3 * np.pi / 4], dtype=np.float32)
    g = geo.Geometry3D(vg, astra.create_proj_geom('cone', 1.0, 1.0, 8, 8, ang, 40.0, 20.0))
    dirs = [orc.dominant_axis3d(orc.CONE, v, 8, 8) for v in g.views_array()]
    assert dirs[0] == 1 and dirs[1] == 0


def test_bp3d_slices_match_z_range(orc):
    """The single-slice BP used by the full-size checks equals the slices of a
    whole-volume BP (cone and parallel)."""
    rng = np.random.default_rng(4)
    ang = np.linspace(0, 2 * np.pi, 9, endpoint=False).astype(np.float32)
    for kind in (orc.CONE, orc.PAR3D):
        if kind == orc.CONE:
            views = orc.cone_views(ang, 20, 18, 60.0, 30.0)
        else:
            views = orc.cone_views(ang, 20, 18, 60.0, 30.0)
            d = views[:, 3:6] + 10 * views[:, 6:9] + 9 * views[:, 9:12] - views[:, 0:3]
            views[:, 0:3] = d / np.linalg.norm(d, axis=1, keepdims=True)
        proj = rng.random((18, 9, 20), dtype=np.float32)
        full = orc.bp3d(kind, views, proj, (12, 14, 16))
        sl = orc.bp3d_slices(kind, views, proj, (12, 14, 16), [0, 5, 11])
        for i, z in enumerate([0, 5, 11]):
            assert np.allclose(sl[i], full[z], rtol=1e-12, atol=1e-12)
