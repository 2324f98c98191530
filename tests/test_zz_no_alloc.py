"""nxs_sgm_device_static: the matcher for callers that must not allocate
device memory (their memory is owned by another allocator, or cudaMalloc's
device synchronisation is too slow for their thread). It keeps its scratch in
one fixed 64 MiB array of the library instead of allocating.

Checked through the C ABI against the allocating entry point, nxs_sgm_device,
bit for bit (tolerance 0, as every disparity test here), on two calls in a row
with different pairs and settings, so a call cannot lean on what the one before
it left in the shared array. This file is collected last; it passes alone in a
fresh process and after the other tests.
"""
import ctypes

import numpy as np
import pytest

from tests import gpu_util as g

pytestmark = pytest.mark.gpu


def _static_entry(native):
    fn = native.load().nxs_sgm_device_static
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32,
                   ctypes.POINTER(native.SgmParams), ctypes.c_void_p, ctypes.c_void_p,
                   ctypes.c_char_p, ctypes.c_size_t]
    return fn


def test_no_alloc_matcher_equals_the_allocating_one_on_two_calls_in_a_row():
    from nx_stereo_b200 import native, scene

    entry = _static_entry(native)
    ctx = native.Context(0)
    cases = [((364, 272), dict(disparities=64, paths=8), 1),
             ((97, 31), dict(disparities=128, paths=3, p1=10, p2=60, stage_mask=True), 2)]
    inputs, static_out = [], []
    for (w, h), settings, seed in cases:  # the two calls, back to back
        left, right = scene.rectified_pair(w, h, seed=seed, rectangles=6, max_disparity=56)
        d_left, d_right = g.dev(left), g.dev(right)
        d_out = g.empty((h, w), g.torch().float32)
        params = native.sgm_params(**settings)
        error = ctypes.create_string_buffer(512)
        status = entry(g.ptr(d_left), g.ptr(d_right), w, h, ctypes.byref(params), g.ptr(d_out),
                       g.stream(), error, 512)
        assert status == native.OK, error.value.decode()
        inputs.append((d_left, d_right, w, h, settings))
        static_out.append(d_out)
    for (d_left, d_right, w, h, settings), d_static in zip(inputs, static_out):
        d_want = g.empty((h, w), g.torch().float32)
        ctx.sgm_device(g.ptr(d_left), g.ptr(d_right), w, h, g.ptr(d_want), g.stream(),
                       **settings)
        assert g.same_bits(g.host(d_static), g.host(d_want))
    ctx.close()


def test_no_alloc_matcher_refuses_pairs_beyond_its_scratch():
    from nx_stereo_b200 import native

    entry = _static_entry(native)
    d_image = g.empty((544, 728), g.torch().uint8)
    d_out = g.empty((544, 728), g.torch().float32)
    params = native.sgm_params(disparities=128, paths=8)
    error = ctypes.create_string_buffer(512)
    status = entry(g.ptr(d_image), g.ptr(d_image), 728, 544, ctypes.byref(params), g.ptr(d_out),
                   g.stream(), error, 512)
    assert status == native.BAD_ARGUMENT
    assert b"64 MiB" in error.value and b"nxs_sgm_device" in error.value
    assert np.isfinite(native.scratch_bytes(728, 544, 128))
