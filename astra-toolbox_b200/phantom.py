"""Seeded synthetic phantoms: random ellipsoids (3D) and ellipses (2D).

The workloads the projection core is measured on are synthetic: volumes of
additive random ellipsoids / ellipses with numpy.random.Generator(PCG64(seed))
parameters.  Generation runs in torch on the requested device.
"""
import numpy as np
import torch


def _rotation(rng):
    q, r = np.linalg.qr(rng.normal(size=(3, 3)))
    q = q * np.sign(np.diag(r))
    if np.linalg.det(q) < 0:
        q[:, 0] = -q[:, 0]
    return q


def ellipsoid_params(n, shape, seed, axes=(20.0, 200.0), inner=0.8):
    """n ellipsoids for a (z, y, x) volume: centres uniform in the inner
    fraction of the volume, semi-axes uniform in `axes` (voxels), uniform random
    orientation, intensities uniform in [0, 1]."""
    rng = np.random.Generator(np.random.PCG64(seed))
    nz, ny, nx = shape
    ext = np.array([nx, ny, nz], dtype=np.float64)
    out = []
    for _ in range(n):
        c = (rng.uniform(-0.5, 0.5, 3) * inner) * ext
        a = rng.uniform(axes[0], axes[1], 3)
        R = _rotation(rng)
        val = rng.uniform(0.0, 1.0)
        out.append((c, a, R, val))
    return out


def ellipsoids(shape, n=12, seed=0, axes=(20.0, 200.0), device="cpu", dtype=torch.float32):
    """(z, y, x) volume of n additive random ellipsoids (voxel units, centred grid)."""
    nz, ny, nx = shape
    vol = torch.zeros(shape, dtype=torch.float32, device=device)
    x = torch.arange(nx, device=device, dtype=torch.float32) - 0.5 * nx + 0.5
    y = torch.arange(ny, device=device, dtype=torch.float32) - 0.5 * ny + 0.5
    params = ellipsoid_params(n, shape, seed, axes)
    for (c, a, R, val) in params:
        Rt = torch.tensor(R, dtype=torch.float32, device=device)
        # process slab by slab to bound temporary memory
        for z0 in range(0, nz, 64):
            z1 = min(nz, z0 + 64)
            z = torch.arange(z0, z1, device=device, dtype=torch.float32) - 0.5 * nz + 0.5
            Z, Y, X = torch.meshgrid(z, y, x, indexing="ij")
            d = torch.stack((X - c[0], Y - c[1], Z - c[2]), dim=-1)
            loc = d @ Rt  # coordinates in the ellipsoid frame
            q = (loc[..., 0] / a[0]) ** 2 + (loc[..., 1] / a[1]) ** 2 + (loc[..., 2] / a[2]) ** 2
            vol[z0:z1] += (q <= 1.0).to(torch.float32) * float(val)
    return vol.to(dtype)


def ellipses(shape, n=10, seed=0, axes=(10.0, 80.0), device="cpu", dtype=torch.float32):
    """(rows, cols) image of n additive random ellipses: centres uniform in the
    inner 80 %, semi-axes uniform in `axes` pixels, rotation uniform in [0, pi),
    intensities uniform in [0, 1]."""
    rng = np.random.Generator(np.random.PCG64(seed))
    H, W = shape
    img = torch.zeros(shape, dtype=torch.float32, device=device)
    x = torch.arange(W, device=device, dtype=torch.float32) - 0.5 * W + 0.5
    y = torch.arange(H, device=device, dtype=torch.float32) - 0.5 * H + 0.5
    Y, X = torch.meshgrid(y, x, indexing="ij")
    for _ in range(n):
        cx, cy = rng.uniform(-0.4, 0.4, 2) * np.array([W, H])
        a, b = rng.uniform(axes[0], axes[1], 2)
        th = rng.uniform(0.0, np.pi)
        v = rng.uniform(0.0, 1.0)
        ct, st = np.cos(th), np.sin(th)
        u = (X - cx) * ct + (Y - cy) * st
        w = -(X - cx) * st + (Y - cy) * ct
        img += ((u / a) ** 2 + (w / b) ** 2 <= 1.0).to(torch.float32) * float(v)
    return img.to(dtype)
