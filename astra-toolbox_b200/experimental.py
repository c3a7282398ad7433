"""astra.experimental: direct projection calls (python/astra/experimental.pyx).

direct_FP3D / direct_BP3D take a 'cuda3d' projector id and the volume and
projection data as numpy arrays or torch tensors (torch CUDA tensors are used
in place, like the reference's DLPack / GPULink path; host arrays are copied
to the device and the result copied back).
"""
from . import _lib
from . import data as _d
from . import projector as _P

MODE_ADD = _lib.MODE_ADD
MODE_SET = _lib.MODE_SET


def _projector(projector_id):
    pr = _d.lookup(projector_id)
    if not isinstance(pr, _P.Projector3D):
        raise _lib.AstraError(1, "Not a cuda3d projector: %r" % (projector_id,))
    return pr


def direct_FPBP3D(projector_id, vol, proj, mode, t):
    """Forward ('FP') or backward ('BP') projection with SET or ADD semantics
    (experimental.pyx:172-203)."""
    pr = _projector(projector_id)
    if t == "FP":
        _P.fp3d(pr, vol, proj, mode=mode)
    elif t == "BP":
        _P.bp3d(pr, vol, proj, mode=mode)
    else:
        raise _lib.AstraError(1, "t must be 'FP' or 'BP'")


def direct_FP3D(projector_id, vol, proj):
    """proj = A vol (experimental.pyx:205-215)."""
    direct_FPBP3D(projector_id, vol, proj, MODE_SET, "FP")


def direct_BP3D(projector_id, vol, proj):
    """vol = B proj (experimental.pyx:217-227)."""
    direct_FPBP3D(projector_id, vol, proj, MODE_SET, "BP")


def accumulate_FP(projector_id, vol_id, proj_id):
    """proj += A vol on data ids (experimental.pyx accumulate_FP)."""
    pr = _projector(projector_id)
    v = _d.lookup(vol_id, _d.DataObject)
    p = _d.lookup(proj_id, _d.DataObject)
    if v.tensor.is_cuda and p.tensor.is_cuda:
        pr.fp(v.tensor, p.tensor, mode=MODE_ADD)
    else:
        _P.fp3d_host(pr, v.tensor, p.tensor, mode=MODE_ADD)
    p.changed()


def accumulate_BP(projector_id, vol_id, proj_id):
    """vol += B proj on data ids (experimental.pyx accumulate_BP)."""
    pr = _projector(projector_id)
    v = _d.lookup(vol_id, _d.DataObject)
    p = _d.lookup(proj_id, _d.DataObject)
    if v.tensor.is_cuda and p.tensor.is_cuda:
        pr.bp(p.tensor, v.tensor, mode=MODE_ADD)
    else:
        _P.bp3d_host(pr, p.tensor, v.tensor, mode=MODE_ADD)
    v.changed()


def accumulate_FDK(projector_id, vol_id, proj_id, short_scan=False):
    """vol += FDK(proj) on data ids (experimental.pyx accumulate_FDK)."""
    pr = _projector(projector_id)
    v = _d.lookup(vol_id, _d.DataObject)
    p = _d.lookup(proj_id, _d.DataObject)
    if v.tensor.is_cuda and p.tensor.is_cuda:
        _P.fdk(pr, p.tensor, v.tensor, short_scan=short_scan, mode=MODE_ADD)
    else:
        _P.fdk_host(pr, p.tensor, v.tensor, short_scan=short_scan, mode=MODE_ADD)
    v.changed()
