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


def _call(name, *args):
    error = ctypes.create_string_buffer(512)
    fn = getattr(lib(), name)
    fn.restype = ctypes.c_int
    status = fn(*args, error, 512)
    if status != 0:
        raise RuntimeError(error.value.decode())


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def rectify(frame, k, d, inverse_pr, size):
    """Stage.Rectification's rectify.comp (lib/nx_stereo/kernels.ex:49-83) for
    one u8 frame and camera, to `size` = (height, width)."""
    frame = np.ascontiguousarray(frame, np.uint8)
    fh, fw = frame.shape
    h, w = size
    camera = np.ascontiguousarray(np.concatenate([np.ravel(k), np.ravel(d), np.ravel(inverse_pr)]),
                                  np.float32)
    out = np.empty((h, w), np.uint8)
    _call("nxs_ref_rectify", _p(frame), fw, fh, _p(camera), w, h, _p(out))
    return out


def despeckle(disparity, min_support=12.0, max_diff=1.0):
    """Stage.SpeckleFilter's despeckle.comp (kernels.ex:114-134), radius 3."""
    disparity = np.ascontiguousarray(disparity, np.float32)
    h, w = disparity.shape
    out = np.empty_like(disparity)
    _call("nxs_ref_despeckle", _p(disparity), w, h, ctypes.c_float(min_support),
          ctypes.c_float(max_diff), _p(out))
    return out


def temporal(current, previous, missed, alpha=0.4, delta=2.0, hold=2.0):
    """Stage.TemporalFilter's temporal_filter.comp (kernels.ex:168-189):
    (filtered, missed_out)."""
    current, previous, missed = (np.ascontiguousarray(a, np.float32)
                                 for a in (current, previous, missed))
    filtered, missed_out = np.empty_like(current), np.empty_like(current)
    _call("nxs_ref_temporal", _p(current), _p(previous), _p(missed), current.size,
          ctypes.c_float(alpha), ctypes.c_float(delta), ctypes.c_float(hold), _p(filtered),
          _p(missed_out))
    return filtered, missed_out


def depth(disparity, focal_length_px, baseline_m):
    """Stage.Depth's depth.comp (kernels.ex:191-212): (depth_mm, depth_m)."""
    disparity = np.ascontiguousarray(disparity, np.float32)
    mm = np.empty(disparity.shape, np.uint16)
    m = np.empty_like(disparity)
    _call("nxs_ref_depth", _p(disparity), disparity.size, ctypes.c_float(focal_length_px),
          ctypes.c_float(baseline_m), _p(mm), _p(m))
    return mm, m


def point_cloud(depth_m, decimation, focal_length_px, cx, cy, nearest_m=0.05, farthest_m=20.0):
    """Stage.PointCloud's point_cloud_rows.comp + column_sums.comp
    (kernels.ex:214-245): (grid, kept)."""
    depth_m = np.ascontiguousarray(depth_m, np.float32)
    h, w = depth_m.shape
    grid = np.empty((h // decimation, w // decimation, 3), np.float32)
    kept = np.zeros(1, np.float32)
    _call("nxs_ref_point_cloud", _p(depth_m), w, h, decimation, ctypes.c_float(focal_length_px),
          ctypes.c_float(cx), ctypes.c_float(cy), ctypes.c_float(nearest_m),
          ctypes.c_float(farthest_m), _p(grid), _p(kept))
    return grid, int(kept[0])


def quality(current, previous):
    """Stage.Quality's disparity_rows.comp + column_sums.comp (kernels.ex:247-268):
    the five sums."""
    current = np.ascontiguousarray(current, np.float32)
    previous = np.ascontiguousarray(previous, np.float32)
    h, w = current.shape
    sums = np.zeros(5, np.float32)
    _call("nxs_ref_quality", _p(current), _p(previous), w, h, _p(sums))
    return sums


WINDOWS = {"sparse_9x7": 0, "dense_9x5": 1, "dense_9x5_blend": 2}


def sgm_band(left, right, base, disparities=128, paths=8, band=16, census="sparse_9x7", p1=8,
             p2=64, uniqueness=1.0526315789473684, subgroup_size=32):
    """NxStereo.sgm_band/4 (lib/nx_stereo.ex:282-321) as the reference's band
    pipeline (lib/nx_stereo/vulkan.ex:196-255) computes it."""
    left = np.ascontiguousarray(left, np.uint8)
    right = np.ascontiguousarray(right, np.uint8)
    base = np.ascontiguousarray(base, np.int32)
    h, w = left.shape
    out = np.empty((h, w), np.float32)
    _call("nxs_ref_sgm_band", _p(left), _p(right), _p(base), w, h, disparities, paths, band,
          WINDOWS[census], ctypes.c_float(p1), ctypes.c_float(p2), ctypes.c_float(uniqueness),
          _p(out), subgroup_size)
    return out


def sgm_coarse_to_fine(left, right, paths=8, coarse_paths=None, band=16, margin=4,
                       fine_census="sparse_9x7", p1=8, p2=64, uniqueness=1.0526315789473684,
                       subgroup_size=32, with_base=False):
    """NxStereo.sgm_coarse_to_fine/3 (lib/nx_stereo.ex:160-225) as the
    reference's shaders compute it: shrink, the coarse sgm/3, the band bases
    and the band pipeline."""
    left = np.ascontiguousarray(left, np.uint8)
    right = np.ascontiguousarray(right, np.uint8)
    h, w = left.shape
    out = np.empty((h, w), np.float32)
    base = np.empty((h, w), np.int32)
    _call("nxs_ref_sgm_coarse_to_fine", _p(left), _p(right), w, h, paths, coarse_paths or paths,
          band, margin, WINDOWS[fine_census], ctypes.c_float(p1), ctypes.c_float(p2),
          ctypes.c_float(uniqueness), _p(out), _p(base), subgroup_size)
    return (out, base) if with_base else out
