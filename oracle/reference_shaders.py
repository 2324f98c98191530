"""ctypes access to the reference's own shaders run on the CPU
(oracle/_ref/libnxs_ref_shaders.so, built by oracle/build_ref.py).

TEST INFRASTRUCTURE ONLY: it checks the oracle against the reference itself
and produces the reference fixtures under tests/golden/. The library exists
where the reference checkout was present when it was built (oracle/_ref/ is
git-ignored); `available()` says whether it is there.
"""
import ctypes
import os

import numpy as np

from . import build_ref as _build

_lib = None
_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")


def available():
    return os.path.exists(_build.LIBRARY) or os.path.isdir(_build.SHADERS)


def lib():
    global _lib
    if _lib is None:
        path = _build.LIBRARY if not os.path.isdir(_build.SHADERS) else _build.build()
        L = ctypes.CDLL(path)
        L.nxs_ref_sgm.restype = ctypes.c_int
        L.nxs_ref_sgm.argtypes = [_u8p, _u8p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                  ctypes.c_int, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                  ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                  ctypes.c_char_p, ctypes.c_int]
        _lib = L
    return _lib


def sgm(left, right, disparities=64, paths=8, p1=8, p2=64, uniqueness=1.0526315789473684,
        subgroup_size=32, with_selection=False):
    """NxStereo.sgm/3 (lib/nx_stereo.ex:64-74) as the reference's shader
    pipeline (lib/nx_stereo/vulkan.ex:262-333) computes it. With
    `with_selection`, also the selection's disparity and keys before the
    left-right check."""
    left = np.ascontiguousarray(left, np.uint8)
    right = np.ascontiguousarray(right, np.uint8)
    h, w = left.shape
    out = np.empty((h, w), np.float32)
    selected = np.empty((h, w), np.float32)
    keys = np.empty((h, w), np.uint32)
    error = ctypes.create_string_buffer(512)
    status = lib().nxs_ref_sgm(left, right, w, h, disparities, paths, float(p1), float(p2),
                               float(uniqueness), out.ctypes.data, selected.ctypes.data,
                               keys.ctypes.data, subgroup_size, error, 512)
    if status != 0:
        raise RuntimeError(error.value.decode())
    return (out, selected, keys) if with_selection else out
