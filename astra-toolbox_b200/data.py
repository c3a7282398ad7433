"""Data objects and the id registry behind data2d / data3d / projector /
algorithm (the reference's CData3DManager / CAstraIndexManager,
python/astra/data3d_c.pyx, data2d_c.pyx).

A data object holds a float32 torch tensor on the GPU (the reference keeps
float32 host memory and copies it to the GPU per call; here the data stay
resident), or, for 3D data beyond the device memory budget (gpu.py), in
pinned host memory, streamed through the GPUs per call.  Linked numpy arrays are mirrored on the device and written back
after every operation that changes them; linked torch CUDA tensors, and CUDA
arrays of other libraries passed through DLPack, are used in place (zero
copy).
"""
import itertools

import numpy as np
import torch

from ._lib import AstraError
from . import geometry as G
from . import gpu as _gpu

_ids = itertools.count(1)
_objects = {}


def new_id():
    return next(_ids)


def register(obj):
    i = new_id()
    _objects[i] = obj
    return i


def lookup(i, cls=None):
    obj = _objects.get(int(i))
    if obj is None or (cls is not None and not isinstance(obj, cls)):
        raise AstraError(1, "Unknown object id %r" % (i,))
    return obj


def remove(i):
    _objects.pop(int(i), None)


def ids_of(cls):
    return [i for i, o in _objects.items() if isinstance(o, cls)]


def _device():
    return torch.device("cuda", torch.cuda.current_device())


class DataObject:
    """'-vol' or '-sino' / '-proj3d' data with its geometry."""

    def __init__(self, kind, geometry, dims3):
        self.kind = kind  # 'vol' or 'sino'
        self.geometry = geometry
        self.is3d = dims3
        if kind == 'vol':
            self.shape = tuple(G.vol_shape(geometry))
        else:
            self.shape = tuple(G.proj_shape(geometry))
        self.tensor = None
        self.host = None       # linked numpy array (written back after changes)
        self.foreign = False   # linked through DLPack from another library

    def _host_resident(self):
        # 3D data beyond the device budget stays in (pinned) host memory and
        # is streamed through the GPUs by FP3D / BP3D / FDK
        return self.is3d and _gpu.host_resident(self.shape)

    def _empty(self):
        if self._host_resident():
            return torch.empty(self.shape, dtype=torch.float32, pin_memory=torch.cuda.is_available())
        return torch.empty(self.shape, dtype=torch.float32, device=_device())

    def fill(self, data):
        self.tensor = self._empty()
        if data is None:
            self.tensor.zero_()
        elif np.isscalar(data):
            self.tensor.fill_(float(data))
        else:
            arr = data.detach().cpu().numpy() if isinstance(data, torch.Tensor) else np.asarray(data)
            if tuple(arr.shape) != self.shape:
                raise AstraError(1, "The dimensions of the data %s do not match those specified in the geometry %s"
                                 % (tuple(arr.shape), self.shape))
            self.tensor.copy_(torch.from_numpy(np.ascontiguousarray(arr, dtype=np.float32)))

    def link(self, data):
        from .projector import dlpack_tensor
        d, foreign = dlpack_tensor(data)
        if foreign:
            # another library's array (CuPy, JAX, ...): used in place through
            # DLPack; results are synchronised in changed()
            self.foreign = True
            data = d
        if isinstance(data, torch.Tensor):
            if tuple(data.shape) != self.shape:
                raise AstraError(1, "The dimensions of the data do not match those specified in the geometry")
            if data.dtype != torch.float32:
                raise AstraError(1, "Linked data must be float32")
            if not data.is_contiguous():
                raise AstraError(1, "Linked data must be contiguous")
            if data.is_cuda:
                self.tensor = data
                return
            self.host = data.numpy()
        else:
            if not isinstance(data, np.ndarray) or data.dtype != np.float32:
                raise AstraError(1, "Linked data must be a float32 numpy array or torch tensor")
            if not data.flags['C_CONTIGUOUS']:
                raise AstraError(1, "Linked data must be C-contiguous")
            if not data.flags['WRITEABLE']:
                raise AstraError(1, "Linked data must be writeable")
            if tuple(data.shape) != self.shape:
                raise AstraError(1, "The dimensions of the data do not match those specified in the geometry")
            self.host = data
        if self._host_resident():
            # streamed from the linked host array itself (no device mirror)
            self.tensor = torch.from_numpy(self.host)
            self.host = None
            return
        self.tensor = torch.from_numpy(self.host).to(_device())

    def changed(self):
        """Write device data back to a linked host array; for data linked
        through DLPack from another library, wait for the writes so that
        library's streams see them."""
        if self.host is not None:
            self.host[...] = self.tensor.cpu().numpy()
        elif self.foreign and self.tensor.is_cuda:
            torch.cuda.current_stream(self.tensor.device).synchronize()

    def get(self):
        return self.tensor.cpu().numpy()

    def store(self, data):
        if np.isscalar(data):
            self.tensor.fill_(float(data))
        else:
            arr = data.detach().cpu().numpy() if isinstance(data, torch.Tensor) else np.asarray(data)
            if tuple(arr.shape) != self.shape:
                raise AstraError(1, "The dimensions of the data do not match those specified in the geometry")
            self.tensor.copy_(torch.from_numpy(np.ascontiguousarray(arr, dtype=np.float32)))
        self.changed()


def create(datatype, geometry, data=None, link=False, dims3=True):
    if datatype == '-vol':
        kind = 'vol'
    elif datatype in ('-sino', '-proj3d', '-sinocone'):
        kind = 'sino'
    else:
        raise ValueError("Invalid datatype. Please specify '-vol' or '-proj3d'")
    obj = DataObject(kind, geometry, dims3)
    if link:
        obj.link(data)
    else:
        obj.fill(data)
    return register(obj)
