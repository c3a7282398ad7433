"""Geometry conversion (host code, CPU): libb2tomo's per-view vectors are
bit-identical to the reference's convertAstraGeometry for all nine geometry
types, against the committed fixtures (tests/golden/make_geometry_golden.py)
and, when the reference build is present, against it directly."""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
FIXTURE = os.path.join(HERE, "golden", "geometry_views.npz")


def _cases():
    import make_geometry_golden as mg
    return mg.cases()


@pytest.mark.parametrize("i", range(5))
def test_3d_views_bit_exact_vs_fixture(geo, i):
    c3, _ = _cases()
    name, vg, pg = c3[i]
    g = geo.Geometry3D(vg, pg)
    d = np.load(FIXTURE)
    assert np.array_equal(g.views_array(), d[name + "_views"]), name
    assert np.array_equal(np.array(g.vol_scale, dtype=np.float32), d[name + "_scale"]), name


@pytest.mark.parametrize("i", range(4))
def test_2d_views_bit_exact_vs_fixture(geo, i):
    _, c2 = _cases()
    name, vg, pg = c2[i]
    g = geo.Geometry2D(vg, pg)
    d = np.load(FIXTURE)
    assert np.array_equal(g.views_array(), d[name + "_views"]), name
    assert np.float32(g.output_scale) == d[name + "_scale"][0], name


def test_against_reference_build_directly(geo):
    from oracle import ref
    if not ref.available():
        pytest.skip("reference build not present")
    c3, c2 = _cases()
    for name, vg, pg in c3:
        v, s = ref.geom3d(vg, pg)
        assert np.array_equal(geo.Geometry3D(vg, pg).views_array(), v), name
    for name, vg, pg in c2:
        v, s = ref.geom2d(vg, pg)
        assert np.array_equal(geo.Geometry2D(vg, pg).views_array(), v), name


def test_non_square_pixels_refused(astra, geo):
    vg = astra.create_vol_geom(10, 12, -5.0, 5.0, -7.0, 7.0)
    pg = astra.create_proj_geom('parallel', 1.0, 16, np.array([0.0], dtype=np.float32))
    with pytest.raises(astra.AstraError):
        geo.Geometry2D(vg, pg)
