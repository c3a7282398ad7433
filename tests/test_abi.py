"""The C ABI library loads and exports every entry point include/b2tomo.h declares
(no compute calls: these run without a GPU)."""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = [os.path.join(ROOT, "include", f) for f in sorted(os.listdir(os.path.join(ROOT, "include")))
           if f.endswith(".h")]


def declared_functions():
    names = []
    for h in HEADERS:
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_]*\s*\*?\s*(b2t_[a-z0-9_]+)\s*\(", src, flags=re.M)
    return sorted(set(names))


def test_header_declares_functions():
    names = declared_functions()
    assert "b2t_fp3d" in names and "b2t_bp3d" in names and len(names) >= 10


def test_library_exports_every_declared_symbol(astra):
    lib = astra.load_library()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_header(astra):
    from importlib import import_module
    L = import_module("astra-toolbox_b200._lib")
    assert set(declared_functions()) <= set(L.SIGNATURES), set(declared_functions()) - set(L.SIGNATURES)


def test_host_only_calls_without_gpu(astra):
    """Geometry entry points are host code and run here; bad args give a status."""
    L = __import__("importlib").import_module("astra-toolbox_b200._lib")
    lib = L.load()
    assert lib.b2t_version() >= 100
    views = (L.View3D * 2)()
    ang = np.array([0.0, 1.0], dtype=np.float32)
    assert lib.b2t_cone_views(2, 4, 4, 10.0, 5.0, 1.0, 1.0, ang.ctypes.data, views) == 0
    assert lib.b2t_cone_views(2, 4, 4, 10.0, 5.0, 1.0, 1.0, None, views) == L.B2T_OK + 1
    assert b"null" in lib.b2t_last_error()
    # invalid geometry is rejected before any device work
    g = L.Geom3D(7, L.Dims3D(4, 4, 4, 2, 4, 4), (ctypes.c_float * 3)(1, 1, 1), views)
    p = L.Params3D(1, 1, 1.0, 0)
    assert lib.b2t_fp3d(ctypes.byref(g), ctypes.byref(p), 16, 0, 16, 0, 0, 1, None) == 1
    g.kind = 2
    g.dims.vol_x = 0
    assert lib.b2t_bp3d(ctypes.byref(g), ctypes.byref(p), 16, 0, 16, 0, 0, 1, None) == 1
    assert lib.b2t_vec_op(99, None, None, None, 0.0, 4, None) == 1
