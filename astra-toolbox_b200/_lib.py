"""ctypes binding of libb2tomo (the C ABI declared in include/b2tomo.h).

The shared library is built in-tree (csrc/Makefile -> libb2tomo.so next to this
file).  There is no fallback: if the library is missing or fails to load,
every projector call raises.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libb2tomo.so")

# status codes (b2tomo.h)
B2T_OK = 0
STATUS_NAMES = {
    0: "OK", 1: "INVALID_ARG", 2: "UNSUPPORTED", 3: "CUDA", 4: "NO_MEMORY", 5: "ABORTED", 6: "TIMEOUT",
}

MODE_ADD, MODE_SET = 0, 1
F32, F16, BF16 = 0, 1, 2
GEOM_PAR3D, GEOM_CONE, GEOM_PAR2D, GEOM_FAN2D, GEOM_CYLCONE = 1, 2, 3, 4, 5
KER_DEFAULT, KER_SUM_SQUARE_WEIGHTS, KER_FDK_WEIGHTING, KER_2D_WEIGHTING, KER_MATCHED_BP = 0, 1, 2, 3, 4
FILTER_NONE, FILTER_RAMLAK = 0, 1
# E_FBPFILTER names (src/Filters.cpp:508-532) -> codes, in the reference's order
FILTER_NAMES = ['none', 'ram-lak', 'shepp-logan', 'cosine', 'hamming', 'hann', 'tukey', 'lanczos', 'triangular',
                'gaussian', 'barlett-hann', 'blackman', 'nuttall', 'blackman-harris', 'blackman-nuttall',
                'flat-top', 'kaiser', 'parzen', 'projection', 'sinogram', 'rprojection', 'rsinogram']
FILTER_PROJECTION, FILTER_SINOGRAM, FILTER_RPROJECTION, FILTER_RSINOGRAM = 18, 19, 20, 21


class FilterConfig(ctypes.Structure):
    _fields_ = [("type", ctypes.c_int32), ("d", ctypes.c_float), ("parameter", ctypes.c_float),
                ("custom", ctypes.c_void_p), ("custom_width", ctypes.c_uint32), ("custom_height", ctypes.c_uint32)]
(OP_SET, OP_MUL_SCALAR, OP_MUL, OP_ADD_MUL, OP_ADD_SCALED, OP_SCALE_AND_ADD, OP_INVERT,
 OP_CLAMP_MIN, OP_CLAMP_MAX, OP_ADD) = range(10)


class AstraError(RuntimeError):
    """Raised when a library call fails (the reference raises astra.log.AstraError)."""

    def __init__(self, status, message):
        self.status = status
        super().__init__("%s: %s" % (STATUS_NAMES.get(status, str(status)), message))


class View3D(ctypes.Structure):
    _fields_ = [("src", ctypes.c_double * 3), ("det_s", ctypes.c_double * 3),
                ("det_u", ctypes.c_double * 3), ("det_v", ctypes.c_double * 3)]


class Dims3D(ctypes.Structure):
    _fields_ = [("vol_x", ctypes.c_uint32), ("vol_y", ctypes.c_uint32), ("vol_z", ctypes.c_uint32),
                ("angles", ctypes.c_uint32), ("det_u", ctypes.c_uint32), ("det_v", ctypes.c_uint32)]


class Geom3D(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("dims", Dims3D), ("vol_scale", ctypes.c_float * 3),
                ("views", ctypes.POINTER(View3D))]


class View3DCyl(ctypes.Structure):
    _fields_ = [("src", ctypes.c_double * 3), ("det_c", ctypes.c_double * 3), ("det_u", ctypes.c_double * 3),
                ("det_v", ctypes.c_double * 3), ("radius", ctypes.c_double)]


class Geom3DCyl(ctypes.Structure):
    _fields_ = [("dims", Dims3D), ("vol_scale", ctypes.c_float * 3), ("views", ctypes.POINTER(View3DCyl))]


class StreamConfig(ctypes.Structure):
    _fields_ = [("device_bytes", ctypes.c_size_t), ("n_devices", ctypes.c_uint32),
                ("devices", ctypes.POINTER(ctypes.c_int32))]


class Params3D(ctypes.Structure):
    _fields_ = [("det_supersample", ctypes.c_uint32), ("voxel_supersample", ctypes.c_uint32),
                ("output_scale", ctypes.c_float), ("kernel", ctypes.c_int32)]


class VolGeom3D(ctypes.Structure):
    _fields_ = [("cols", ctypes.c_uint32), ("rows", ctypes.c_uint32), ("slices", ctypes.c_uint32),
                ("min_x", ctypes.c_float), ("max_x", ctypes.c_float), ("min_y", ctypes.c_float),
                ("max_y", ctypes.c_float), ("min_z", ctypes.c_float), ("max_z", ctypes.c_float)]


class View2D(ctypes.Structure):
    _fields_ = [("src", ctypes.c_float * 2), ("det_s", ctypes.c_float * 2), ("det_u", ctypes.c_float * 2)]


class Dims2D(ctypes.Structure):
    _fields_ = [("vol_width", ctypes.c_uint32), ("vol_height", ctypes.c_uint32),
                ("angles", ctypes.c_uint32), ("dets", ctypes.c_uint32)]


class Geom2D(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("dims", Dims2D), ("output_scale", ctypes.c_float),
                ("views", ctypes.POINTER(View2D))]


class VolGeom2D(ctypes.Structure):
    _fields_ = [("cols", ctypes.c_uint32), ("rows", ctypes.c_uint32), ("min_x", ctypes.c_float),
                ("max_x", ctypes.c_float), ("min_y", ctypes.c_float), ("max_y", ctypes.c_float)]


class Problem2D(ctypes.Structure):
    _fields_ = [("geom", Geom2D), ("det_supersample", ctypes.c_uint32), ("pixel_supersample", ctypes.c_uint32)]


class Problem3D(ctypes.Structure):
    _fields_ = [("geom", Geom3D), ("det_supersample", ctypes.c_uint32), ("output_scale", ctypes.c_float)]


ALGO_SIRT, ALGO_CGLS, ALGO_SART = 1, 2, 3


class AlgoOptions(ctypes.Structure):
    _fields_ = [("relaxation", ctypes.c_float), ("use_min", ctypes.c_int32), ("min_value", ctypes.c_float),
                ("use_max", ctypes.c_int32), ("max_value", ctypes.c_float), ("vol_mask", ctypes.c_void_p),
                ("sino_mask", ctypes.c_void_p), ("min_mask", ctypes.c_void_p), ("max_mask", ctypes.c_void_p)]


_P = ctypes.c_void_p
_SZ = ctypes.c_size_t
_I32 = ctypes.c_int32
_U32 = ctypes.c_uint32
_F = ctypes.c_float

# name -> (restype, argtypes); every entry point declared in include/b2tomo.h
SIGNATURES = {
    "b2t_last_error": (ctypes.c_char_p, []),
    "b2t_version": (_I32, []),
    "b2t_kernel_launches": (ctypes.c_uint64, []),
    "b2t_set_device": (_I32, [_I32]),
    "b2t_device_errors": (_I32, [_P]),
    "b2t_bp_path_stats": (_I32, [_P]),
    "b2t_fp_path_stats": (_I32, [_P]),
    "b2t_matched_path_stats": (_I32, [_P]),
    "b2t_cone_views": (_I32, [_U32, _U32, _U32, _F, _F, _F, _F, _P, _P]),
    "b2t_par3d_views": (_I32, [_U32, _U32, _U32, _F, _F, _P, _P]),
    "b2t_vec_views3d": (_I32, [_U32, _U32, _U32, _P, _P]),
    "b2t_normalize_views3d": (_I32, [_P, _I32, _U32, _P, _P]),
    "b2t_par_views": (_I32, [_U32, _U32, _F, _P, _P]),
    "b2t_fan_views": (_I32, [_U32, _U32, _F, _F, _F, _P, _P]),
    "b2t_vec_views2d": (_I32, [_U32, _U32, _P, _P]),
    "b2t_normalize_views2d": (_I32, [_P, _I32, _U32, _P, _P]),
    "b2t_fp3d": (_I32, [_P, _P, _P, _SZ, _P, _SZ, _I32, _I32, _P]),
    "b2t_bp3d": (_I32, [_P, _P, _P, _SZ, _P, _SZ, _I32, _I32, _P]),
    "b2t_normalize_views3d_cyl": (_I32, [_P, _U32, _P, _P]),
    "b2t_fp3d_host": (_I32, [_P, _P, _P, _P, _I32, _P]),
    "b2t_bp3d_host": (_I32, [_P, _P, _P, _P, _I32, _P]),
    "b2t_fdk_host": (_I32, [_P, _P, _I32, ctypes.c_float, _P, _P, _I32, _P]),
    "b2t_stream_plan": (_I32, [_I32, _P, _P, _P, _P]),
    "b2t_fp3d_cyl": (_I32, [_P, _P, _P, _SZ, _P, _SZ, _I32, _P]),
    "b2t_bp3d_cyl": (_I32, [_P, _P, _P, _SZ, _P, _SZ, _I32, _P]),
    "b2t_fp2d": (_I32, [_P, _U32, _P, _SZ, _P, _SZ, _I32, _P]),
    "b2t_bp2d": (_I32, [_P, _U32, _I32, _P, _SZ, _P, _SZ, _I32, _P]),
    "b2t_fdk": (_I32, [_P, _P, _I32, _F, _P, _SZ, _P, _SZ, _I32, _I32, _P]),
    "b2t_fdk_weight_filter": (_I32, [_P, _P, _I32, _P, _SZ, _I32, _P]),
    "b2t_filter_rows": (_I32, [_P, _SZ, _U32, _SZ, _P, _P]),
    "b2t_filter_taps": (_I32, [_P, _U32, _U32, _P, _P]),
    "b2t_fbp2d": (_I32, [_P, _P, _I32, _P, _SZ, _P, _SZ, _I32, _P]),
    "b2t_algo_create3d": (_I32, [_I32, _P, _P, _P, _P]),
    "b2t_algo_create3d_cyl": (_I32, [_I32, _P, _P, _P, _P]),
    "b2t_algo_create2d": (_I32, [_I32, _P, _U32, _U32, _P, _P]),
    "b2t_algo_run": (_I32, [_P, _P, _P, _I32, _I32, _P]),
    "b2t_algo_residual_norm": (_I32, [_P, _P, _P, _P, _P]),
    "b2t_algo_set_projection_order": (_I32, [_P, _P, _U32]),
    "b2t_algo_abort": (None, [_P]),
    "b2t_algo_destroy": (None, [_P]),
    "b2t_vec_op": (_I32, [_I32, _P, _P, _P, _F, _SZ, _P]),
    "b2t_dot_f64": (_I32, [_P, _P, _SZ, _I32, _P, _P]),
    "b2t_dot_f64_noalloc": (_I32, [_P, _P, _SZ, _I32, _P, _P]),
    "b2t_onchip_peak": (_I32, [_I32, _P]),
    "b2t_debug_fail_alloc": (_I32, [ctypes.c_int64, _P]),
    "b2t_debug_live_allocations": (ctypes.c_int64, []),
    "b2t_selftest_bounded_wait": (_I32, [_I32, ctypes.c_uint64, _P]),
    "b2t_release_cached_memory": (_I32, []),
    "b2t_autotune_fp3d": (_I32, [_P, _P, _P, _SZ, _P, _SZ, _I32, _P, _P]),
    "b2t_autotune_bp3d": (_I32, [_P, _P, _P, _SZ, _P, _SZ, _I32, _P, _P]),
    "b2t_batch2d_create": (_I32, [_P, _I32, _P]),
    "b2t_batch2d_layout": (_I32, [_P, _P, _P, _P, _P]),
    "b2t_batch2d_fp": (_I32, [_P, _P, _P, _I32, _P]),
    "b2t_batch2d_bp": (_I32, [_P, _P, _P, _I32, _P]),
    "b2t_algo_create_batch2d": (_I32, [_I32, _P, _P, _P]),
    "b2t_batch2d_destroy": (None, [_P]),
    "b2t_batch3d_create": (_I32, [_P, _I32, _P]),
    "b2t_batch3d_layout": (_I32, [_P, _P, _P, _P, _P]),
    "b2t_batch3d_fp": (_I32, [_P, _P, _P, _I32, _P]),
    "b2t_batch3d_bp": (_I32, [_P, _P, _P, _I32, _P]),
    "b2t_batch3d_matched_bp": (_I32, [_P, _P, _P, _I32, _P]),
    "b2t_batch3d_destroy": (None, [_P]),
}

_lib = None


def load(path=LIB_PATH):
    """Load libb2tomo.so and declare every signature; raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise AstraError(3, "libb2tomo.so not built at %s (run __graft_entry__.build())" % path)
    lib = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(status):
    if status != B2T_OK:
        msg = load().b2t_last_error()
        raise AstraError(status, msg.decode() if msg else "")


def call(name, *args):
    """Call a status-returning entry point and raise AstraError on failure."""
    check(getattr(load(), name)(*args))


def ptr(a):
    """Raw pointer of a numpy array / ctypes object / torch tensor / int."""
    if a is None:
        return None
    if isinstance(a, int):
        return a
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    return ctypes.addressof(a)
