"""Convenience creators (python/astra/creators.py): sinograms, backprojections,
reconstructions and projectors through the GPU path."""
from . import algorithm as _alg
from . import data2d as _d2
from . import data3d as _d3
from . import projector as _P
from ._lib import AstraError
from .geometry import create_proj_geom, create_vol_geom  # noqa: F401


def create_projector(proj_type, proj_geom, vol_geom, options=None):
    """create_projector (creators.py:488-520): 'cuda' or 'cuda3d'."""
    return _P.create({'type': proj_type, 'ProjectionGeometry': proj_geom, 'VolumeGeometry': vol_geom,
                      'options': options or {}})


def create_sino3d_gpu(data, proj_geom, vol_geom, returnData=True, gpuIndex=None):
    """create_sino3d_gpu (creators.py:361-400): FP3D_CUDA of data (array or id)."""
    vol_id = data if isinstance(data, int) else _d3.create('-vol', vol_geom, data)
    sino_id = _d3.create('-sino', proj_geom, 0)
    cfg = _alg.astra_dict('FP3D_CUDA')
    cfg['VolumeDataId'] = vol_id
    cfg['ProjectionDataId'] = sino_id
    if gpuIndex is not None:
        cfg['option']['GPUIndex'] = gpuIndex
    alg = _alg.create(cfg)
    _alg.run(alg)
    _alg.delete(alg)
    if not isinstance(data, int):
        _d3.delete(vol_id)
    if returnData:
        return sino_id, _d3.get(sino_id)
    return sino_id


def create_backprojection3d_gpu(data, proj_geom, vol_geom, returnData=True, gpuIndex=None):
    """create_backprojection3d_gpu (creators.py:450-485): BP3D_CUDA of data."""
    sino_id = data if isinstance(data, int) else _d3.create('-sino', proj_geom, data)
    vol_id = _d3.create('-vol', vol_geom, 0)
    cfg = _alg.astra_dict('BP3D_CUDA')
    cfg['ProjectionDataId'] = sino_id
    cfg['ReconstructionDataId'] = vol_id
    if gpuIndex is not None:
        cfg['option']['GPUIndex'] = gpuIndex
    alg = _alg.create(cfg)
    _alg.run(alg)
    _alg.delete(alg)
    if not isinstance(data, int):
        _d3.delete(sino_id)
    if returnData:
        return vol_id, _d3.get(vol_id)
    return vol_id


def create_sino(data, proj_id, returnData=True, gpuIndex=None):
    """create_sino (creators.py:297-340) with a 'cuda' projector."""
    pr = _P.lookup_projector(proj_id)
    vol_id = data if isinstance(data, int) else _d2.create('-vol', pr.vol_geom, data)
    sino_id = _d2.create('-sino', pr.proj_geom, 0)
    cfg = _alg.astra_dict('FP_CUDA')
    cfg['ProjectorId'] = proj_id
    cfg['VolumeDataId'] = vol_id
    cfg['ProjectionDataId'] = sino_id
    alg = _alg.create(cfg)
    _alg.run(alg)
    _alg.delete(alg)
    if not isinstance(data, int):
        _d2.delete(vol_id)
    if returnData:
        return sino_id, _d2.get(sino_id)
    return sino_id


def create_backprojection(data, proj_id, returnData=True):
    """create_backprojection (creators.py:403-447) with a 'cuda' projector."""
    pr = _P.lookup_projector(proj_id)
    sino_id = data if isinstance(data, int) else _d2.create('-sino', pr.proj_geom, data)
    vol_id = _d2.create('-vol', pr.vol_geom, 0)
    cfg = _alg.astra_dict('BP_CUDA')
    cfg['ProjectorId'] = proj_id
    cfg['ProjectionDataId'] = sino_id
    cfg['ReconstructionDataId'] = vol_id
    alg = _alg.create(cfg)
    _alg.run(alg)
    _alg.delete(alg)
    if not isinstance(data, int):
        _d2.delete(sino_id)
    if returnData:
        return vol_id, _d2.get(vol_id)
    return vol_id


def create_reconstruction(rec_type, proj_id, sinogram, iterations=1, use_mask='no', mask=None,
                          use_minc='no', minc=0, use_maxc='no', maxc=255, returnData=True):
    """create_reconstruction (creators.py:523-590) for the CUDA algorithms."""
    if not rec_type.endswith('_CUDA'):
        raise AstraError(2, "Only the _CUDA reconstruction algorithms are provided")
    pr = _P.lookup_projector(proj_id)
    is3d = isinstance(pr, _P.Projector3D)
    dm = _d3 if is3d else _d2
    sino_id = sinogram if isinstance(sinogram, int) else dm.create('-sino', pr.proj_geom, sinogram)
    rec_id = dm.create('-vol', pr.vol_geom, 0)
    cfg = _alg.astra_dict(rec_type)
    cfg['ProjectorId'] = proj_id
    cfg['ProjectionDataId'] = sino_id
    cfg['ReconstructionDataId'] = rec_id
    if use_mask == 'yes':
        cfg['option']['ReconstructionMaskId'] = mask if isinstance(mask, int) else dm.create('-vol', pr.vol_geom, mask)
    if use_minc == 'yes':
        cfg['option']['MinConstraint'] = minc
    if use_maxc == 'yes':
        cfg['option']['MaxConstraint'] = maxc
    alg = _alg.create(cfg)
    _alg.run(alg, iterations)
    _alg.delete(alg)
    if not isinstance(sinogram, int):
        dm.delete(sino_id)
    if returnData:
        return rec_id, dm.get(rec_id)
    return rec_id
