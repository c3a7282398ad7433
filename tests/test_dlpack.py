"""DLPack interchange (python/astra/utils.pyx:237-260 getDLPackCapsule): data
from another library is used in place, and the consumer's stream is passed to
the producer's __dlpack__ (the reference leaves that argument unused)."""
import importlib

import numpy as np
import pytest

torch = pytest.importorskip("torch")


class Foreign:
    """A stand-in for another array library: exposes only the DLPack protocol
    over a torch tensor and records the stream it is asked for."""

    def __init__(self, t):
        self.t = t
        self.streams = []

    def __dlpack__(self, stream=None, **kwargs):
        self.streams.append(stream)
        return self.t.__dlpack__()

    def __dlpack_device__(self):
        return self.t.__dlpack_device__()


def _P():
    return importlib.import_module("astra-toolbox_b200.projector")


def test_foreign_host_data_shares_memory():
    P = _P()
    base = torch.arange(12, dtype=torch.float32).reshape(3, 4)
    t, foreign = P.dlpack_tensor(Foreign(base))
    assert foreign
    t[1, 2] = -5.0
    assert base[1, 2] == -5.0
    assert P.dlpack_tensor(base) == (None, False)
    assert P.dlpack_tensor(np.zeros(3, np.float32)) == (None, False)
    cap = torch.ones(4).__dlpack__()
    t2, foreign2 = P.dlpack_tensor(cap)
    assert foreign2 and float(t2.sum()) == 4.0
    with pytest.raises(Exception):
        P.as_device_tensor(object(), "cpu")


@pytest.mark.gpu
def test_direct_fp_bp_on_foreign_cuda_arrays(astra):
    ang = np.linspace(0, 2 * np.pi, 20, endpoint=False).astype(np.float32)
    vg = astra.create_vol_geom(24, 26, 20)
    pg = astra.create_proj_geom('cone', 1.0, 1.0, 24, 30, ang, 100.0, 50.0)
    pid = astra.create_projector('cuda3d', pg, vg)
    pr = _P().Projector3D(pg, vg)
    vol = torch.rand(pr.vol_shape, device='cuda')
    want = torch.zeros(pr.proj_shape, device='cuda')
    pr.fp(vol, want)
    fv, fp = Foreign(vol), Foreign(torch.full(pr.proj_shape, 3.0, device='cuda'))
    astra.experimental.direct_FP3D(pid, fv, fp)
    assert torch.equal(fp.t, want)
    # the producer was handed the consumer's stream (DLPack: 1 = legacy default)
    cur = torch.cuda.current_stream().cuda_stream
    assert fp.streams and fp.streams[-1] in (cur, 1)
    back = Foreign(torch.zeros(pr.vol_shape, device='cuda'))
    astra.experimental.direct_BP3D(pid, back, Foreign(want))
    ref = torch.zeros(pr.vol_shape, device='cuda')
    pr.bp(want, ref)
    assert torch.equal(back.t, ref)


@pytest.mark.gpu
def test_linked_foreign_array_is_updated_in_place(astra):
    ang = np.linspace(0, np.pi, 30, endpoint=False).astype(np.float32)
    vg = astra.create_vol_geom(32, 32)
    pg = astra.create_proj_geom('parallel', 1.0, 48, ang)
    pr = astra.Projector2D(pg, vg)
    x = torch.rand(pr.vol_shape, device='cuda')
    b = torch.zeros(pr.proj_shape, device='cuda')
    pr.fp(x, b)
    rec = Foreign(torch.zeros(pr.vol_shape, device='cuda'))
    sid = astra.data2d.link('-sino', pg, Foreign(b))
    rid = astra.data2d.link('-vol', vg, rec)
    cfg = astra.astra_dict('SIRT_CUDA')
    cfg['ProjectionDataId'] = sid
    cfg['ReconstructionDataId'] = rid
    aid = astra.algorithm.create(cfg)
    astra.algorithm.run(aid, 20)
    assert float(rec.t.abs().sum()) > 0.0
    assert torch.equal(rec.t.cpu(), torch.from_numpy(astra.data2d.get(rid)))
    astra.algorithm.delete(aid)
    astra.data2d.delete([sid, rid])
