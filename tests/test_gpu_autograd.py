"""Differentiable projector (exact adjoint) on the GPU: dot-product test,
gradient check against central finite differences, and the deviation of
ASTRA's unmatched BP used as a gradient (workload shape of the par3d
differentiable configuration at reduced size)."""
import importlib

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _setup(astra, n=40, na=36, nd=48, kind='parallel3d'):
    ang = np.linspace(0, np.pi, na, endpoint=False).astype(np.float32)
    vg = astra.create_vol_geom(n, n, n)
    if kind == 'parallel3d':
        pg = astra.create_proj_geom('parallel3d', 1.0, 1.0, nd, nd, ang)
    else:
        pg = astra.create_proj_geom('cone', 1.0, 1.0, nd, nd, ang * 2, 4.0 * n, 2.0 * n)
    return astra.Projector3D(pg, vg)


def _tv(x, eps=1e-8):
    dz = x[1:, :-1, :-1] - x[:-1, :-1, :-1]
    dy = x[:-1, 1:, :-1] - x[:-1, :-1, :-1]
    dx = x[:-1, :-1, 1:] - x[:-1, :-1, :-1]
    return torch.sqrt(dx * dx + dy * dy + dz * dz + eps).sum()


@pytest.mark.parametrize("kind", ["parallel3d", "cone"])
def test_dot_product(astra, kind):
    AG = importlib.import_module("astra-toolbox_b200.autograd")
    pr = _setup(astra, kind=kind)
    g = torch.Generator(device='cuda').manual_seed(0)
    # <A x, y> = <x, A^T y> up to FP32 rounding.  With signed data the dot
    # products cancel to a small fraction of their terms, so the rounding of
    # the two operators (which sum in different orders) is measured against
    # the sum of the terms' magnitudes; with non-negative data there is no
    # cancellation and the plain relative difference is tight.
    for signed in (True, False):
        if signed:
            x = torch.randn(pr.vol_shape, device='cuda', generator=g)
            y = torch.randn(pr.proj_shape, device='cuda', generator=g)
        else:
            x = torch.rand(pr.vol_shape, device='cuda', generator=g)
            y = torch.rand(pr.proj_shape, device='cuda', generator=g)
        ax = AG.forward_project(x, pr)
        aty = AG.back_project(y, pr)
        lhs = float((ax.double() * y.double()).sum())
        rhs = float((x.double() * aty.double()).sum())
        if signed:
            scale = float((ax.double() * y.double()).abs().sum())
            assert abs(lhs - rhs) / scale < 1e-6
        else:
            assert abs(lhs - rhs) / abs(lhs) < 2e-6


def test_gradient_vs_finite_differences(astra):
    AG = importlib.import_module("astra-toolbox_b200.autograd")
    ph = importlib.import_module("astra-toolbox_b200.phantom")
    pr = _setup(astra)
    x_true = ph.ellipsoids(pr.vol_shape, 6, seed=1, axes=(4.0, 14.0), device='cuda')
    b = AG.forward_project(x_true, pr).detach()
    gen = torch.Generator(device='cuda').manual_seed(3)
    b = b + 0.01 * float(b.max()) * torch.randn(b.shape, device='cuda', generator=gen)
    x = (x_true + 0.1 * torch.randn(x_true.shape, device='cuda', generator=gen)).requires_grad_(True)

    def loss_fn(v):
        r = AG.forward_project(v, pr) - b
        return (r.double() ** 2).sum() + 1e-3 * _tv(v.double())

    loss = loss_fn(x)
    loss.backward()
    grad = x.grad.detach()
    rng = np.random.default_rng(0)
    idx = [tuple(int(rng.integers(5, s - 5)) for s in pr.vol_shape) for _ in range(64)]
    errs = []
    with torch.no_grad():
        for p in idx:
            h = 1e-2
            xp = x.detach().clone()
            xp[p] += h
            xm = x.detach().clone()
            xm[p] -= h
            fd = (float(loss_fn(xp)) - float(loss_fn(xm))) / (2 * h)
            errs.append(abs(fd - float(grad[p])) / max(1e-6, abs(fd)))
    assert np.median(errs) < 1e-3 and np.max(errs) < 2e-2, (np.median(errs), np.max(errs))


@pytest.mark.parametrize("kind", ["parallel3d", "cone"])
def test_astra_bp_gradient_deviation_is_reported(astra, orc, kind):
    """ASTRA's BP is an approximate adjoint: its deviation from the exact
    adjoint on white noise is large for cone beams (the 1/den^2 weight is not
    the ray-length weight) but the directions agree.  The GPU deviation must
    equal the FP64 oracle's on the same input."""
    AG = importlib.import_module("astra-toolbox_b200.autograd")
    pr = _setup(astra, kind=kind)
    r_np = np.random.default_rng(5).standard_normal(pr.proj_shape).astype(np.float32)
    r = torch.from_numpy(r_np).cuda()
    exact = AG.back_project(r, pr)
    approx = AG.astra_bp_gradient(pr, r)
    dev = float(torch.linalg.vector_norm(approx - exact) / torch.linalg.vector_norm(exact))
    cos = float((approx.double() * exact.double()).sum()
                / (torch.linalg.vector_norm(approx.double()) * torch.linalg.vector_norm(exact.double())))
    G = pr.geom
    views = G.views_array()
    o_ex = orc.fp3d_transpose(G.kind, views, r_np, pr.vol_shape, G.vol_scale)
    o_ap = orc.bp3d(G.kind, views, r_np, pr.vol_shape, G.vol_scale)
    o_dev = float(np.linalg.norm(o_ap - o_ex) / np.linalg.norm(o_ex))
    assert abs(dev - o_dev) < 2e-3 * max(1.0, o_dev), (dev, o_dev)
    assert dev > 1e-4 and cos > 0.85, (dev, cos)


def test_batched_and_half(astra):
    AG = importlib.import_module("astra-toolbox_b200.autograd")
    pr = _setup(astra, n=24, na=12, nd=28)
    x = torch.rand((2,) + pr.vol_shape, device='cuda')
    y = AG.forward_project(x, pr)
    assert y.shape == (2,) + pr.proj_shape
    assert torch.allclose(y[1], AG.forward_project(x[1], pr))
    xh = x[0].to(torch.bfloat16).requires_grad_(True)
    yh = AG.forward_project(xh, pr)
    yh.float().sum().backward()
    assert xh.grad is not None and xh.grad.dtype == torch.bfloat16


@pytest.mark.parametrize("kind", ["parallel3d", "cone"])
def test_batch_dimension_is_one_launch_each_way(astra, kind):
    """A leading batch dimension of small float32 items is projected in one
    persistent launch (b2t_batch3d_fp) and its gradient in one more (the
    exact adjoint b2t_batch3d_matched_bp): the pair passes the dot-product
    test, and each item matches the single-problem projectors to rounding."""
    AG = importlib.import_module("astra-toolbox_b200.autograd")
    lib = importlib.import_module("astra-toolbox_b200._lib").load()
    pr = _setup(astra, n=32, na=20, nd=40, kind=kind)
    x = torch.rand((3,) + pr.vol_shape, device='cuda', requires_grad=True)
    n0 = lib.b2t_kernel_launches()
    y = AG.forward_project(x, pr)
    torch.cuda.synchronize()
    assert lib.b2t_kernel_launches() - n0 == 1
    g = torch.rand_like(y)
    n0 = lib.b2t_kernel_launches()
    (y * g).sum().backward()
    torch.cuda.synchronize()
    assert lib.b2t_kernel_launches() - n0 == 1
    lhs = float((y.detach().double() * g.double()).sum())
    rhs = float((x.detach().double() * x.grad.double()).sum())
    assert abs(lhs - rhs) / abs(lhs) < 1e-5, (lhs, rhs)
    for i in range(3):
        yi = AG.forward_project(x[i].detach(), pr)
        assert float((y[i].detach() - yi).norm() / yi.norm()) < 2e-6
        gi = AG._at(pr, g[i])
        assert float((x.grad[i] - gi).norm() / gi.norm()) < 2e-5
