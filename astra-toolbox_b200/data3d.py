"""astra.data3d: 3D volume and projection data objects (python/astra/data3d.py)."""
from . import data as _d
from . import geometry as _G


def create(datatype, geometry, data=None):
    """Create a '-vol' or '-proj3d' object filled with a scalar or an array."""
    return _d.create(datatype, geometry, data, dims3=True)


def link(datatype, geometry, data):
    """Link a float32 numpy array, torch tensor or DLPack object (CUDA data
    zero-copy)."""
    return _d.create(datatype, geometry, data, link=True, dims3=True)


def get(i):
    return _d.lookup(i, _d.DataObject).get()


def get_shared(i):
    """The data as a torch tensor sharing the device memory of the object."""
    return _d.lookup(i, _d.DataObject).tensor


def get_geometry(i):
    return _d.lookup(i, _d.DataObject).geometry


def change_geometry(i, geometry):
    obj = _d.lookup(i, _d.DataObject)
    shape = _G.vol_shape(geometry) if obj.kind == 'vol' else _G.proj_shape(geometry)
    if tuple(shape) != obj.shape:
        raise ValueError("The dimensions of the data %s do not match those specified in the geometry %s"
                         % (obj.shape, tuple(shape)))
    obj.geometry = geometry


def store(i, data):
    _d.lookup(i, _d.DataObject).store(data)


def dimensions(i):
    return _d.lookup(i, _d.DataObject).shape


def delete(ids):
    for i in (ids if isinstance(ids, (list, tuple)) else [ids]):
        _d.remove(i)


def clear():
    for i in _d.ids_of(_d.DataObject):
        _d.remove(i)


def info():
    for i in _d.ids_of(_d.DataObject):
        o = _d.lookup(i)
        print("%d\t%s\t%s" % (i, o.kind, o.shape))
