"""Angle-sharded operators and SIRT (astra-toolbox_b200.parallel) on CPU:
world_size 2 over gloo, each rank projecting its block of views with the FP64
oracle.  The sharded FP must equal the rows of the unsharded FP, the sharded
BP the full BP, and sharded SIRT the single-process SIRT."""
import importlib
import os
import socket
import tempfile

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402


class OracleOp:
    """FP / BP of one (sub-)geometry through the FP64 oracle, on CPU tensors."""

    def __init__(self, proj_geom, vol_geom):
        from oracle import oracle as orc
        G = importlib.import_module("astra-toolbox_b200.geometry").Geometry3D(vol_geom, proj_geom)
        self.orc = orc
        self.kind = 2 if G.kind == 2 else 1
        self.views = G.views_array()
        self.vs = G.vol_scale
        self.vol_shape = G.vol_shape
        self.proj_shape = G.proj_shape

    def fp(self, vol, proj):
        nv, na, nu = self.proj_shape
        out = self.orc.fp3d(self.kind, self.views, vol.numpy().astype(np.float32), nu, nv, self.vs)
        proj.copy_(torch.from_numpy(np.asarray(out, dtype=np.float32)))

    def bp(self, proj, vol):
        out = self.orc.bp3d(self.kind, self.views, proj.numpy().astype(np.float32), self.vol_shape, self.vs)
        vol.copy_(torch.from_numpy(np.asarray(out, dtype=np.float32)))


def _geoms(kind):
    astra = importlib.import_module("astra-toolbox_b200")
    vg = astra.create_vol_geom(14, 16, 12)
    ang = np.linspace(0, 2 * np.pi, 21, endpoint=False).astype(np.float32)
    if kind == "cone":
        pg = astra.create_proj_geom('cone', 1.0, 1.0, 16, 20, ang, 60.0, 30.0)
    else:
        pg = astra.create_proj_geom('parallel3d', 1.0, 1.0, 16, 20, ang[:13])
    return pg, vg


def _phantom(shape):
    rng = np.random.default_rng(3)
    v = rng.random(shape, dtype=np.float32)
    v[:, :, : shape[2] // 2] += 1.0
    return torch.from_numpy(v)


def _worker(rank, world, port, kind, out_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        par = importlib.import_module("astra-toolbox_b200.parallel")
        pg, vg = _geoms(kind)
        op = par.AngleShardedOperator(pg, vg, projector_factory=OracleOp)
        x_true = _phantom(op.vol_shape)
        b_local = torch.empty(op.proj_shape)
        op.fp(x_true, b_local)
        back = torch.empty(op.vol_shape)
        op.bp(b_local, back)
        sirt = par.ShardedSIRT(op, relaxation=0.9, min_constraint=0.0)
        x = torch.zeros(op.vol_shape)
        sirt.run(b_local, x, 4)
        res = sirt.residual_norm(b_local, x)
        np.savez(os.path.join(out_dir, "rank%d.npz" % rank), b_local=b_local.numpy(), back=back.numpy(),
                 x=x.numpy(), res=res, start=op.start, stop=op.stop)
    finally:
        dist.barrier()
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_view_range_partitions():
    par = importlib.import_module("astra-toolbox_b200.parallel")
    for n in (1, 7, 21, 720):
        for world in (1, 2, 3, 8):
            blocks = [par.view_range(n, world, r) for r in range(world)]
            assert blocks[0][0] == 0 and blocks[-1][1] == n
            assert all(blocks[i][1] == blocks[i + 1][0] for i in range(world - 1))
            sizes = [b - a for a, b in blocks]
            assert max(sizes) - min(sizes) <= 1


@pytest.mark.parametrize("kind", ["cone", "parallel3d"])
def test_sharded_operators_and_sirt_world2(kind):
    par = importlib.import_module("astra-toolbox_b200.parallel")
    with tempfile.TemporaryDirectory() as d:
        mp.start_processes(_worker, args=(2, _free_port(), kind, d), nprocs=2, join=True, start_method="spawn")
        r = [np.load(os.path.join(d, "rank%d.npz" % k)) for k in range(2)]
    # single process, same code path (no process group): the reference result
    pg, vg = _geoms(kind)
    full = par.AngleShardedOperator(pg, vg, projector_factory=OracleOp)
    assert (full.start, full.stop) == (0, full.proj_shape[1])
    x_true = _phantom(full.vol_shape)
    b = torch.empty(full.proj_shape)
    full.fp(x_true, b)
    back = torch.empty(full.vol_shape)
    full.bp(b, back)
    sirt = par.ShardedSIRT(full, relaxation=0.9, min_constraint=0.0)
    x = torch.zeros(full.vol_shape)
    sirt.run(b, x, 4)
    res = sirt.residual_norm(b, x)
    # FP: each rank holds its rows of the full projections
    for k in range(2):
        s0, s1 = int(r[k]["start"]), int(r[k]["stop"])
        assert np.array_equal(r[k]["b_local"], b.numpy()[:, s0:s1, :])
    # BP and SIRT: every rank holds the full (replicated) result
    for k in range(2):
        assert np.allclose(r[k]["back"], back.numpy(), rtol=1e-5, atol=1e-5 * float(back.abs().max()))
        err = np.linalg.norm(r[k]["x"] - x.numpy()) / np.linalg.norm(x.numpy())
        assert err < 1e-5, err
        assert abs(float(r[k]["res"]) - res) <= 1e-5 * res
    assert np.array_equal(r[0]["x"], r[1]["x"]), "replicas must stay identical"
