"""The C-ABI library loads and exports every symbol include/*.h declares.

CPU only: no compute calls, and context creation is allowed to fail with
RTB200_E_DEVICE where there is no GPU.
"""
import ctypes
import glob
import os
import re

import numpy as np
import pytest

from rise_b200 import _native, raycaster

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"\b(rtb200_[a-z0-9_]+)\s*\(", src):
            names.add(m.group(1))
    return sorted(names)


def test_headers_declare_entry_points():
    names = declared_functions()
    assert "rtb200_cast_closest" in names and "rtb200_scene_commit" in names
    assert len(names) >= 15


@pytest.mark.parametrize("name", declared_functions())
def test_symbol_exported(name):
    lib = ctypes.CDLL(_native.LIB_PATH)
    assert hasattr(lib, name), name


def test_binding_covers_header():
    assert set(declared_functions()) <= set(_native.SIGNATURES)


def test_invalid_arguments_rejected_without_device():
    L = _native.lib()
    assert L.rtb200_ctx_create(0, 0, None) == _native.E_INVALID
    assert L.rtb200_scene_commit(None, 0) == _native.E_INVALID
    assert L.rtb200_cast_closest(None, None, 0, None) == _native.E_INVALID
    assert L.rtb200_bvh_host_build(None, 5, 0, ctypes.byref(ctypes.c_void_p())) == _native.E_INVALID
    assert L.rtb200_bvh_host_destroy(None) == _native.E_INVALID


def test_struct_layouts():
    assert raycaster.RAY_DTYPE.itemsize == 32
    assert raycaster.HIT_DTYPE.itemsize == 16
    assert raycaster.NODE2_DTYPE.itemsize == 32
    assert raycaster.NODE4_DTYPE.itemsize == 128
    assert np.dtype(raycaster.RAY_DTYPE).names[3] == "tmin"
