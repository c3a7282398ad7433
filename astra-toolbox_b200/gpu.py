"""GPU selection and the device-memory budget (python/astra/astra.py
set_gpu_index / get_gpu_info; the reference's CompositeGeometryManager reads
the budget, src/CompositeGeometryManager.cpp:1409-1477).

set_gpu_index(idx, memory) selects the GPU (or list of GPUs) and a per-GPU
memory budget in bytes (0: no budget).  With a budget, and for any 3D data
larger than half the free device memory, data objects live in pinned host
memory and FP3D / BP3D / FDK stream them through the GPUs in z-slabs and
angle blocks (b2t_fp3d_host, b2t_bp3d_host, b2t_fdk_host).
"""
import ctypes

import numpy as np
import torch

from . import _lib

_gpus = None   # list of device ordinals, or None for the current device
_memory = 0    # per-GPU budget in bytes, 0 = none


def set_gpu_index(idx, memory=0):
    """Select the GPU(s) used and, optionally, a per-GPU memory budget."""
    global _gpus, _memory
    ids = [int(i) for i in (idx if isinstance(idx, (list, tuple)) else [idx])]
    if not ids:
        raise _lib.AstraError(1, "set_gpu_index: empty GPU list")
    if torch.cuda.is_available():
        n = torch.cuda.device_count()
        for i in ids:
            if i < 0 or i >= n:
                raise _lib.AstraError(1, "set_gpu_index: no GPU %d" % i)
        torch.cuda.set_device(ids[0])
    _gpus = ids
    _memory = int(memory)


def get_gpu_info(idx=-1):
    """One line describing GPU idx (-1: the current one), or 'Invalid device'."""
    if not torch.cuda.is_available():
        return "Invalid device"
    if idx < 0:
        idx = torch.cuda.current_device()
    if idx >= torch.cuda.device_count():
        return "Invalid device"
    p = torch.cuda.get_device_properties(idx)
    return "GPU #%d: %s, compute capability %d.%d, %d MB" % (idx, p.name, p.major, p.minor,
                                                              p.total_memory // (1024 * 1024))


def memory_budget():
    return _memory


def stream_config():
    """The b2t_stream_config of the current settings (kept alive by the caller)."""
    ids = _gpus or []
    arr = (ctypes.c_int32 * max(1, len(ids)))(*ids) if ids else None
    cfg = _lib.StreamConfig(ctypes.c_size_t(_memory), len(ids),
                            ctypes.cast(arr, ctypes.POINTER(ctypes.c_int32)) if arr is not None else None)
    cfg._devices = arr  # keep the array alive with the struct
    return cfg


def host_resident(shape):
    """Whether a float32 array of this shape should live in host memory:
    with a memory budget set, or when it exceeds half the free memory of the
    current GPU."""
    if _memory > 0:
        return True
    if not torch.cuda.is_available():
        return False
    nbytes = int(np.prod(shape)) * 4
    free, _ = torch.cuda.mem_get_info()
    return nbytes > free // 2
