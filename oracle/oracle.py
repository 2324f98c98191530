"""ctypes access to the CPU oracle (oracle/_build/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg as the checker. The product (nx_stereo_b200)
never imports it.
"""
import ctypes
import os

import numpy as np

from . import build as _build

_lib = None

_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
_u16p = np.ctypeslib.ndpointer(np.uint16, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_i, _f, _sz = ctypes.c_int, ctypes.c_float, ctypes.c_size_t


class Camera(ctypes.Structure):
    _fields_ = [("k", ctypes.c_float * 9), ("d", ctypes.c_float * 5),
                ("inverse_pr", ctypes.c_float * 9)]


def lib():
    global _lib
    if _lib is None:
        path = _build.build()
        L = ctypes.CDLL(path)
        sig = {
            "oracle_census": (None, [_u8p, _i, _i, _u64p]),
            "oracle_costs": (None, [_u64p, _u64p, _i, _i, _i, _i32p]),
            "oracle_path": (None, [_i32p, _i, _i, _i, _i, _i, _i, _i, _i32p]),
            "oracle_aggregate": (None, [_i32p, _i, _i, _i, _i, _i, _i, _i32p]),
            "oracle_select": (None, [_i32p, _i, _i, _i, _f, _f32p, _u32p]),
            "oracle_consistency": (None, [_f32p, _u32p, _i, _i, _i, _f32p]),
            "oracle_median3": (None, [_f32p, _i, _i, _f32p]),
            "oracle_sgm": (_i, [_u8p, _u8p, _i, _i, _i, _i, _i, _i, _f, _f32p]),
            "oracle_disparity_stage": (_i, [_u8p, _u8p, _i, _i, _i, _i, _i, _i, _f, _f32p]),
            "oracle_rectify": (None, [_u8p, _i, _i, ctypes.POINTER(Camera), _i, _i, _u8p]),
            "oracle_despeckle": (None, [_f32p, _i, _i, _f, _f, _i, _f32p]),
            "oracle_temporal": (None, [_f32p, _f32p, _f32p, _sz, _f, _f, _f, _f]),
            "oracle_depth": (None, [_f32p, _sz, _f, _f, _u16p, _f32p]),
            "oracle_cloud": (ctypes.c_int32, [_f32p, _i, _i, _i, _f, _f, _f, _f, _f, _f32p]),
            "oracle_quality": (None, [_f32p, _f32p, _i, _i, _f32p]),
            "oracle_census_window": (None, [_u8p, _i, _i, _i, _u64p]),
            "oracle_shrink": (None, [_u8p, _i, _i, _u8p]),
            "oracle_band_base": (None, [_f32p, _i, _i, _i, _i, _i32p]),
            "oracle_band_costs": (None, [_u64p, _u64p, _i32p, _i, _i, _i, _i32p]),
            "oracle_band_aggregate": (None, [_i32p, _i32p, _i, _i, _i, _i, _i, _i, _i32p]),
            "oracle_band_select": (None, [_i32p, _i32p, _i, _i, _i, _i, _f, _f32p, _u32p]),
            "oracle_sgm_band": (_i, [_u8p, _u8p, _i32p, _i, _i, _i, _i, _i, _i, _i, _i, _f,
                                     _f32p]),
            "oracle_sgm_coarse_to_fine": (_i, [_u8p, _u8p, _i, _i, _i, _i, _i, _i, _i, _i, _i,
                                               _f, _f32p, ctypes.c_void_p]),
            "oracle_noise": (None, [_i, _i, ctypes.c_uint64, _u8p]),
            "oracle_scene": (None, [_i, _i, ctypes.c_uint64, _u8p, _u8p]),
            "oracle_fast_sgm": (_i, [_u8p, _u8p, _i, _i, _i, _i, _i, _i, _f, _f32p]),
            "oracle_fast_sgm_batch": (_i, [_u8p, _u8p, _i, _i, _i, _i, _i, _i, _i, _f, _f32p, _i]),
            "oracle_fast_pipeline_batch": (ctypes.c_long, [
                _u8p, _u8p, _i, _i, _i, ctypes.POINTER(Camera), ctypes.POINTER(Camera), _i, _i,
                _i, _i, _i, _i, _f, _f, _f, _f, _f, _i, _f, _f, _f, _f, ctypes.c_void_p, _i]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _c(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


def census(image):
    image = _c(image, np.uint8)
    h, w = image.shape
    out = np.empty((h, w), np.uint64)
    lib().oracle_census(image, w, h, out)
    return out


def costs(left_codes, right_codes, disparities):
    h, w = left_codes.shape
    out = np.empty((h, w, disparities), np.int32)
    lib().oracle_costs(_c(left_codes, np.uint64), _c(right_codes, np.uint64), w, h, disparities, out)
    return out


def path(costs_, direction, p1, p2):
    costs_ = _c(costs_, np.int32)
    h, w, d = costs_.shape
    out = np.empty_like(costs_)
    lib().oracle_path(costs_, w, h, d, direction[0], direction[1], p1, p2, out)
    return out


def aggregate(costs_, paths, p1, p2):
    costs_ = _c(costs_, np.int32)
    h, w, d = costs_.shape
    out = np.empty_like(costs_)
    lib().oracle_aggregate(costs_, w, h, d, paths, p1, p2, out)
    return out


def select(sums, uniqueness):
    sums = _c(sums, np.int32)
    h, w, d = sums.shape
    disparity = np.empty((h, w), np.float32)
    keys = np.empty((h, w), np.uint32)
    lib().oracle_select(sums, w, h, d, uniqueness, disparity, keys)
    return disparity, keys


def consistency(disparity, keys, disparities):
    disparity = _c(disparity, np.float32)
    h, w = disparity.shape
    out = np.empty_like(disparity)
    lib().oracle_consistency(disparity, _c(keys, np.uint32), w, h, disparities, out)
    return out


def median3(image):
    image = _c(image, np.float32)
    h, w = image.shape
    out = np.empty_like(image)
    lib().oracle_median3(image, w, h, out)
    return out


def sgm(left, right, disparities=64, paths=8, p1=8, p2=64, uniqueness=1.0526315789473684):
    left, right = _c(left, np.uint8), _c(right, np.uint8)
    h, w = left.shape
    out = np.empty((h, w), np.float32)
    if lib().oracle_sgm(left, right, w, h, disparities, paths, p1, p2, uniqueness, out):
        raise ValueError(f"refused size {w}x{h}")
    return out


def disparity_stage(left, right, disparities=64, paths=8, p1=8, p2=64,
                    uniqueness=1.0526315789473684):
    left, right = _c(left, np.uint8), _c(right, np.uint8)
    h, w = left.shape
    out = np.empty((h, w), np.float32)
    if lib().oracle_disparity_stage(left, right, w, h, disparities, paths, p1, p2, uniqueness, out):
        raise ValueError(f"refused size {w}x{h}")
    return out


def fast_sgm(left, right, disparities=64, paths=8, p1=8, p2=64, uniqueness=1.0526315789473684):
    left, right = _c(left, np.uint8), _c(right, np.uint8)
    h, w = left.shape
    out = np.empty((h, w), np.float32)
    if lib().oracle_fast_sgm(left, right, w, h, disparities, paths, p1, p2, uniqueness, out):
        raise ValueError("refused")
    return out


def fast_sgm_batch(lefts, rights, disparities=128, paths=8, p1=8, p2=64,
                   uniqueness=1.0526315789473684, threads=1):
    lefts, rights = _c(lefts, np.uint8), _c(rights, np.uint8)
    n, h, w = lefts.shape
    out = np.empty((n, h, w), np.float32)
    if lib().oracle_fast_sgm_batch(lefts, rights, n, w, h, disparities, paths, p1, p2,
                                   uniqueness, out, threads):
        raise ValueError("refused")
    return out


def make_camera(k, d, inverse_pr):
    cam = Camera()
    cam.k[:] = [float(v) for v in np.asarray(k, np.float32).ravel()]
    cam.d[:] = [float(v) for v in np.asarray(d, np.float32).ravel()]
    cam.inverse_pr[:] = [float(v) for v in np.asarray(inverse_pr, np.float32).ravel()]
    return cam


def rectify(frame, camera, size):
    frame = _c(frame, np.uint8)
    fh, fw = frame.shape
    h, w = size
    out = np.empty((h, w), np.uint8)
    lib().oracle_rectify(frame, fw, fh, ctypes.byref(camera), w, h, out)
    return out


def despeckle(disparity, min_support=12.0, max_diff=1.0, radius=3):
    disparity = _c(disparity, np.float32)
    h, w = disparity.shape
    out = np.empty_like(disparity)
    lib().oracle_despeckle(disparity, w, h, float(min_support), float(max_diff), radius, out)
    return out


def temporal(current, previous, missed, alpha=0.4, delta=2.0, hold=2.0, max_missed=255.0):
    """Returns (filtered, previous', missed'); inputs are not modified."""
    cur = _c(current, np.float32).copy()
    prev = _c(previous, np.float32).copy()
    miss = _c(missed, np.float32).copy()
    lib().oracle_temporal(cur, prev, miss, cur.size, alpha, delta, hold, max_missed)
    return cur, prev, miss


def depth(disparity, focal_length_px, baseline_m):
    disparity = _c(disparity, np.float32)
    mm = np.empty(disparity.shape, np.uint16)
    m = np.empty(disparity.shape, np.float32)
    lib().oracle_depth(disparity, disparity.size, focal_length_px, baseline_m, mm, m)
    return mm, m


def cloud(depth_m, decimation, focal_length_px, cx, cy, nearest_m=0.05, farthest_m=20.0):
    depth_m = _c(depth_m, np.float32)
    h, w = depth_m.shape
    grid = np.empty((h // decimation, w // decimation, 3), np.float32)
    kept = lib().oracle_cloud(depth_m, w, h, decimation, focal_length_px, cx, cy, nearest_m,
                              farthest_m, grid)
    return grid, int(kept)


def quality(disparity, previous):
    """Returns (sums[5], previous')."""
    disparity = _c(disparity, np.float32)
    prev = _c(previous, np.float32).copy()
    h, w = disparity.shape
    sums = np.empty(5, np.float32)
    lib().oracle_quality(disparity, prev, w, h, sums)
    return sums, prev


def noise(width, height, seed):
    out = np.empty((height, width), np.uint8)
    lib().oracle_noise(width, height, seed, out)
    return out


def scene(width, height, seed):
    left = np.empty((height, width), np.uint8)
    right = np.empty((height, width), np.uint8)
    lib().oracle_scene(width, height, seed, left, right)
    return left, right


def fast_pipeline_batch(left_frames, right_frames, left_camera, right_camera, size,
                        disparities=128, paths=8, p1=8, p2=64, uniqueness=1.0526315789473684,
                        min_support=12.0, max_diff=1.0, focal_length_px=873.0, baseline_m=0.2,
                        decimation=4, principal_point=(364.0, 272.0), nearest_m=0.05,
                        farthest_m=20.0, threads=1, keep_disparities=False):
    """Rectification, matcher, despeckle, depth and cloud per pair on `threads`
    threads. Returns (kept points, disparities or None)."""
    lefts = _c(left_frames, np.uint8)
    rights = _c(right_frames, np.uint8)
    n, fh, fw = lefts.shape
    h, w = size
    out = np.empty((n, h, w), np.float32) if keep_disparities else None
    kept = lib().oracle_fast_pipeline_batch(
        lefts, rights, n, fw, fh, ctypes.byref(left_camera), ctypes.byref(right_camera), w, h,
        disparities, paths, p1, p2, uniqueness, min_support, max_diff, focal_length_px,
        baseline_m, decimation, principal_point[0], principal_point[1], nearest_m, farthest_m,
        out.ctypes.data if out is not None else None, threads)
    if kept < 0:
        raise ValueError("refused")
    return int(kept), out


# ---------------------------------------------------------------- coarse to fine
WINDOWS = {"sparse_9x7": 0, "dense_9x5": 1, "dense_9x5_blend": 2}


def census_window(image, window="sparse_9x7"):
    image = _c(image, np.uint8)
    h, w = image.shape
    out = np.empty((h, w), np.uint64)
    lib().oracle_census_window(image, w, h, WINDOWS[window], out)
    return out


def shrink(image):
    image = _c(image, np.uint8)
    h, w = image.shape
    out = np.empty((h // 2, w // 2), np.uint8)
    lib().oracle_shrink(image, w, h, out)
    return out


def band_base(coarse, band=16, margin=4):
    coarse = _c(coarse, np.float32)
    h, w = coarse.shape
    out = np.empty((2 * h, 2 * w), np.int32)
    lib().oracle_band_base(coarse, w, h, band, margin, out)
    return out


def band_costs(left_codes, right_codes, searched, band):
    h, w = left_codes.shape
    out = np.empty((h, w, band), np.int32)
    lib().oracle_band_costs(_c(left_codes, np.uint64), _c(right_codes, np.uint64),
                            _c(searched, np.int32), w, h, band, out)
    return out


def band_aggregate(costs_, searched, paths, p1, p2):
    costs_ = _c(costs_, np.int32)
    h, w, band = costs_.shape
    out = np.empty_like(costs_)
    lib().oracle_band_aggregate(costs_, _c(searched, np.int32), w, h, band, paths, p1, p2, out)
    return out


def band_select(sums, base, disparities, uniqueness):
    sums = _c(sums, np.int32)
    h, w, band = sums.shape
    disparity = np.empty((h, w), np.float32)
    keys = np.empty((h, w), np.uint32)
    lib().oracle_band_select(sums, _c(base, np.int32), w, h, band, disparities, uniqueness,
                             disparity, keys)
    return disparity, keys


def sgm_band(left, right, base, disparities=128, paths=8, band=16, census="sparse_9x7", p1=8,
             p2=64, uniqueness=1.0526315789473684):
    left, right = _c(left, np.uint8), _c(right, np.uint8)
    h, w = left.shape
    out = np.empty((h, w), np.float32)
    if lib().oracle_sgm_band(left, right, _c(base, np.int32), w, h, disparities, paths, band,
                             WINDOWS[census], p1, p2, uniqueness, out):
        raise ValueError("refused")
    return out


def sgm_coarse_to_fine(left, right, paths=8, coarse_paths=None, band=16, margin=4,
                       fine_census="sparse_9x7", p1=8, p2=64, uniqueness=1.0526315789473684,
                       with_base=False):
    left, right = _c(left, np.uint8), _c(right, np.uint8)
    h, w = left.shape
    out = np.empty((h, w), np.float32)
    base = np.empty((h, w), np.int32)
    if lib().oracle_sgm_coarse_to_fine(left, right, w, h, paths, coarse_paths or paths, band,
                                       margin, WINDOWS[fine_census], p1, p2, uniqueness, out,
                                       base.ctypes.data):
        raise ValueError("refused")
    return (out, base) if with_base else out
