"""astra-toolbox_b200: B200-native drop-in for the ASTRA Toolbox CUDA projection core.

Import with importlib (the directory name is not a Python identifier):

    astra = importlib.import_module("astra-toolbox_b200")

Surface mirrored from the reference (python/astra/__init__.py):
create_vol_geom, create_proj_geom, projector3d / projector ('cuda3d', 'cuda'),
data3d / data2d, algorithm (FP3D_CUDA, BP3D_CUDA, FDK_CUDA, SIRT3D_CUDA,
CGLS3D_CUDA, FP_CUDA, BP_CUDA, SIRT_CUDA, CGLS_CUDA, FBP_CUDA), experimental
(direct_FP3D / direct_BP3D), create_sino3d_gpu / create_backprojection3d_gpu,
create_sino / create_backprojection / create_reconstruction, astra_dict.
Every computation runs in libb2tomo.so (sm_100a); there is no CPU path.
"""
from . import _lib
from ._lib import AstraError
from .geometry import create_proj_geom, create_vol_geom
from .projector import Projector2D, Projector3D
from . import algorithm, batch, data2d, data3d, experimental, projector, projector3d  # noqa: F401
from .batch import Batch2D, Batch3D  # noqa: F401
from .optomo import OpTomo  # noqa: F401
from .gpu import get_gpu_info, set_gpu_index  # noqa: F401
from .algorithm import astra_dict
from .creators import (create_backprojection, create_backprojection3d_gpu, create_projector,  # noqa: F401
                       create_reconstruction, create_sino, create_sino3d_gpu)

__all__ = ["AstraError", "create_proj_geom", "create_vol_geom", "Projector2D", "Projector3D", "algorithm",
           "data2d", "data3d", "experimental", "projector", "projector3d", "astra_dict", "create_projector",
           "create_sino3d_gpu", "create_backprojection3d_gpu", "create_sino", "create_backprojection",
           "create_reconstruction"]


def load_library():
    """Load libb2tomo.so (raises AstraError if it is not built)."""
    return _lib.load()
