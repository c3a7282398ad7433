"""Parity at the sizes the throughput numbers are measured on.

C2 (the bench's cone workload): 512^3 volume of 12 seeded ellipsoids, 720
views over 2 pi, 832^2 detector, SOD 1000, ODD 500.  The whole FP and BP run
on the GPU (the paths that only these sizes reach: 32-bit cell indices over a
136 M-cell array, the BP's 640 + 80 view launches, the circular-orbit fast
path over 512-voxel columns, the tensor-core far taps at 832 columns); the
FP64 oracle checks sampled views of the FP, sampled z-slices of the BP and
sampled views of the FDK filter, 1e-5 relative L2.

C3 (the differentiable par3d workload): 256^3, 360 views over pi, 384^2
detector.  Dot-product test of the exact adjoint (seeded Gaussian x, y, FP64
accumulation) and the gradient of ||FP(x) - b||^2 + 1e-3 TV(x) against
central finite differences at 64 random voxels, b = FP(phantom) + N(0, (0.01
max b)^2).
"""
import importlib

import numpy as np
import pytest

from conftest import rel_l2

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

N, NA, ND, SOD, ODD = 512, 720, 832, 1000.0, 500.0


@pytest.fixture(scope="module")
def c2(astra):
    ph = importlib.import_module("astra-toolbox_b200.phantom")
    ang = np.linspace(0, 2 * np.pi, NA, endpoint=False).astype(np.float32)
    vg = astra.create_vol_geom(N, N, N)
    pg = astra.create_proj_geom('cone', 1.0, 1.0, ND, ND, ang, SOD, ODD)
    pr = astra.Projector3D(pg, vg)
    vol = ph.ellipsoids(pr.vol_shape, 12, seed=0, device='cuda')
    proj = torch.zeros(pr.proj_shape, device='cuda')
    pr.fp(vol, proj)
    back = torch.zeros(pr.vol_shape, device='cuda')
    pr.bp(proj, back)
    torch.cuda.synchronize()
    yield pr, vol, proj, back
    del vol, proj, back
    torch.cuda.empty_cache()


def _sel(n, k):
    return [int(v) for v in np.linspace(0, n - 1, k).round().astype(int)]


def test_c2_fp_full_size_vs_oracle(c2, orc):
    pr, vol, proj, _ = c2
    sel = _sel(NA, 6)
    ref = orc.fp3d(orc.CONE, pr.geom.views_array()[sel], vol.cpu().numpy(), ND, ND, pr.geom.vol_scale)
    got = proj[:, sel, :].double().cpu().numpy()
    for i, a in enumerate(sel):
        assert rel_l2(got[:, i], ref[:, i]) < 1e-5, (a, rel_l2(got[:, i], ref[:, i]))


def test_c2_bp_full_size_vs_oracle(c2, orc):
    pr, _, proj, back = c2
    sl = _sel(N, 4)
    ref = orc.bp3d_slices(orc.CONE, pr.geom.views_array(), proj.cpu().numpy(), pr.vol_shape, sl,
                          pr.geom.vol_scale)
    got = back[sl].double().cpu().numpy()
    for i, z in enumerate(sl):
        assert rel_l2(got[i], ref[i]) < 1e-5, (z, rel_l2(got[i], ref[i]))


def test_c2_fdk_full_size_vs_oracle(c2, orc):
    """FDK at 832 columns (near taps in FP32, far taps on the tensor cores):
    the weighted, filtered projections on sampled views, then the FDK
    backprojection of those filtered projections on sampled slices."""
    P = importlib.import_module("astra-toolbox_b200.projector")
    pr, _, proj, _ = c2
    views = pr.geom.views_array()
    filt = proj.clone()
    P.fdk_weight_filter(pr, filt)
    sel = _sel(NA, 8)
    p = proj[:, sel, :].double().cpu().numpy().copy()
    orc.fdk_weight(p, views[sel])
    p *= len(sel) / float(NA)  # the weight's (pi/2)/n_angles factor, for the full scan
    orc.ramp_filter_rows(p)
    got = filt[:, sel, :].double().cpu().numpy()
    assert rel_l2(got, p) < 1e-5, rel_l2(got, p)
    rec = torch.zeros(pr.vol_shape, device='cuda')
    P.fdk(pr, proj, rec)
    sl = _sel(N, 3)
    ref = orc.bp3d_slices(orc.CONE, views, filt.cpu().numpy(), pr.vol_shape, sl, pr.geom.vol_scale,
                          kernel=orc.KER_FDK)
    got = rec[sl].double().cpu().numpy()
    for i, z in enumerate(sl):
        assert rel_l2(got[i], ref[i]) < 1e-5, (z, rel_l2(got[i], ref[i]))


def _c3(astra):
    ang = np.linspace(0, np.pi, 360, endpoint=False).astype(np.float32)
    vg = astra.create_vol_geom(256, 256, 256)
    pg = astra.create_proj_geom('parallel3d', 1.0, 1.0, 384, 384, ang)
    return astra.Projector3D(pg, vg)


def test_c3_dot_product_full_size(astra):
    AG = importlib.import_module("astra-toolbox_b200.autograd")
    pr = _c3(astra)
    g = torch.Generator(device='cuda').manual_seed(0)
    x = torch.randn(pr.vol_shape, device='cuda', generator=g)
    y = torch.randn(pr.proj_shape, device='cuda', generator=g)
    ax = AG.forward_project(x, pr)
    aty = AG.back_project(y, pr)
    lhs = float((ax.double() * y.double()).sum())
    rhs = float((x.double() * aty.double()).sum())
    scale = float((ax.double() * y.double()).abs().sum())
    # FP32 operators, FP64 accumulation: <Ax, y> = <x, A^T y> to FP32
    # rounding of the operators, measured against the terms' magnitudes
    assert abs(lhs - rhs) / scale < 1e-5, (lhs, rhs, scale)


def test_c3_gradient_vs_finite_differences_full_size(astra):
    AG = importlib.import_module("astra-toolbox_b200.autograd")
    ph = importlib.import_module("astra-toolbox_b200.phantom")
    pr = _c3(astra)
    x_true = ph.ellipsoids(pr.vol_shape, 12, seed=1, axes=(10.0, 100.0), device='cuda')
    b = AG.forward_project(x_true, pr).detach()
    gen = torch.Generator(device='cuda').manual_seed(3)
    b = b + 0.01 * float(b.max()) * torch.randn(b.shape, device='cuda', generator=gen)
    x = (x_true + 0.1 * torch.randn(x_true.shape, device='cuda', generator=gen)).requires_grad_(True)

    def tv(v, eps=1e-8):
        dz = v[1:, :-1, :-1] - v[:-1, :-1, :-1]
        dy = v[:-1, 1:, :-1] - v[:-1, :-1, :-1]
        dx = v[:-1, :-1, 1:] - v[:-1, :-1, :-1]
        return torch.sqrt(dx * dx + dy * dy + dz * dz + eps).sum()

    def loss_fn(v):
        r = AG.forward_project(v, pr) - b
        return (r.double() ** 2).sum() + 1e-3 * tv(v.double())

    loss = loss_fn(x)
    loss.backward()
    grad = x.grad.detach()
    rng = np.random.default_rng(0)
    idx = [tuple(int(rng.integers(8, s - 8)) for s in pr.vol_shape) for _ in range(64)]
    errs = []
    with torch.no_grad():
        xd = x.detach()
        for p in idx:
            h = 1e-2
            xp = xd.clone()
            xp[p] += h
            xm = xd.clone()
            xm[p] -= h
            fd = (float(loss_fn(xp)) - float(loss_fn(xm))) / (2 * h)
            errs.append(abs(fd - float(grad[p])) / max(1e-6, abs(fd)))
    assert np.median(errs) < 1e-3 and np.max(errs) < 2e-2, (np.median(errs), np.max(errs))
