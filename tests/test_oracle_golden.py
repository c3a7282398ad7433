"""The FP64 oracle against golden vectors produced by the reference's own CUDA
build (tests/golden/make_golden.py).  CPU only.

Two bars: the oracle's exact model within 2e-3 relative L2 of the reference
(the reference's texture unit interpolates with 8-bit fractional weights), and
the oracle's tex8 mode (weights rounded to 1/256, as the texture unit does)
within 1e-3.  FDK: the reference filters with cuFFT in float; 2e-3.
sum_square_weights reads no texture: 1e-4.
"""
import glob
import os

import numpy as np
import pytest

from conftest import rel_l2

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FILES = sorted(f for f in glob.glob(os.path.join(GOLDEN, "*.npz"))
               if os.path.basename(f).startswith(("fp", "bp", "fdk", "cyl")))


def _name(f):
    return os.path.basename(f)[:-4]


@pytest.mark.skipif(not FILES, reason="no golden fixtures")
@pytest.mark.parametrize("path", FILES, ids=[_name(f) for f in FILES])
def test_oracle_matches_reference_cuda(orc, path):
    d = np.load(path)
    name = _name(path)
    out = d["output"]
    inp = d["input"]
    views = d["views"]
    rays = 2 if "ss2" in name else 1
    if name.startswith("cyl"):
        # cyl_cone_vec; the matched BP scatters exact weights (no texture)
        vs = d["vol_scale"]
        if name == "cyl_fp":
            nv, na, nu = out.shape
            exact = orc.cylcone_fp(views, inp, nu, nv, vs)
            tex8 = orc.cylcone_fp(views, inp, nu, nv, vs, tex8=True)
        elif name == "cyl_bp":
            exact = orc.cylcone_bp(views, inp, out.shape, vs)
            tex8 = orc.cylcone_bp(views, inp, out.shape, vs, tex8=True)
        else:
            exact = orc.cylcone_fp_transpose(views, inp.astype(np.float64), out.shape, vs)
            assert rel_l2(exact, out) < 1e-5, (name, rel_l2(exact, out))
            return
        assert rel_l2(exact, out) < 2e-3, (name, rel_l2(exact, out))
        assert rel_l2(tex8, out) < 1e-3, (name, rel_l2(tex8, out))
        return
    if "sumsqw" in name:
        # no texture in this kernel: the reference differs from the FP64
        # model only by its float position stepping
        nv, na, nu = out.shape
        exact = orc.par3d_sumsqw(views, tuple(d["vol_shape"]), nu, nv, d["vol_scale"])
        assert rel_l2(exact, out) < 1e-4, (name, rel_l2(exact, out))
        return
    if name.startswith("fp3d"):
        nv, na, nu = out.shape
        kind = int(d["kind"])
        exact = orc.fp3d(kind, views, inp, nu, nv, d["vol_scale"], rays=rays)
        tex8 = orc.fp3d(kind, views, inp, nu, nv, d["vol_scale"], rays=rays, tex8=True)
    elif name.startswith("bp3d"):
        ker = 3 if "2dw" in name else (2 if "fdkw" in name else 0)
        kind = int(d["kind"])
        exact = orc.bp3d(kind, views, inp, out.shape, d["vol_scale"], kernel=ker, rays=rays)
        tex8 = orc.bp3d(kind, views, inp, out.shape, d["vol_scale"], kernel=ker, rays=rays, tex8=True)
    elif name.startswith("fdk"):
        exact = orc.fdk(views, inp, out.shape, d["vol_scale"], short_scan="short" in name)
        tex8 = exact
    elif name.startswith("fp2d"):
        f = orc.fan_fp if int(d["kind"]) == 4 else orc.par_fp
        exact = f(views, inp, out.shape[1], float(d["out_scale"]))
        tex8 = f(views, inp, out.shape[1], float(d["out_scale"]), tex8=True)
    elif name.startswith("bp2d"):
        if int(d["kind"]) == 4:
            fbp = "fbp" in name
            exact = orc.fan_bp(views, inp, out.shape, float(d["out_scale"]), fbp=fbp)
            tex8 = orc.fan_bp(views, inp, out.shape, float(d["out_scale"]), fbp=fbp, tex8=True)
        else:
            exact = orc.par_bp(views, inp, out.shape, float(d["out_scale"]))
            tex8 = orc.par_bp(views, inp, out.shape, float(d["out_scale"]), tex8=True)
    else:
        pytest.skip("unknown fixture")
    assert rel_l2(exact, out) < 2e-3, (name, rel_l2(exact, out))
    assert rel_l2(tex8, out) < 1e-3, (name, rel_l2(tex8, out))
