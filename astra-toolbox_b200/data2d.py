"""astra.data2d: 2D image and sinogram data objects (python/astra/data2d.py)."""
from . import data as _d
from .data3d import change_geometry, delete, dimensions, get, get_geometry, get_shared, info, store  # noqa: F401


def create(datatype, geometry, data=None):
    """Create a '-vol' or '-sino' object filled with a scalar or an array."""
    return _d.create(datatype, geometry, data, dims3=False)


def link(datatype, geometry, data):
    return _d.create(datatype, geometry, data, link=True, dims3=False)


def clear():
    for i in _d.ids_of(_d.DataObject):
        if not _d.lookup(i).is3d:
            _d.remove(i)
