"""The fused entry points equal the steps they fuse, bit for bit: both sides'
rectification in one launch, both images' census in one launch, and the
left-right check with the median in one pass (at the sizes the matcher's
tests use, a row narrower than the 3x3 window, and a 4096-wide image)."""
import ctypes

import numpy as np
import pytest

from tests import gpu_util as g

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def native():
    from nx_stereo_b200 import native as n

    n.load()
    return n


def test_rectify_pair(native):
    from nx_stereo_b200 import scene

    torch = g.torch()
    rig = scene.rig(728, 544)
    cams = scene.cameras(rig)
    cameras = [native.make_camera(cams[s]["k"], cams[s]["d"], cams[s]["inverse_pr"])
               for s in ("left", "right")]
    left, right = scene.rectified_pair(728, 544, seed=4)
    lf, rf = scene.raw_frames(left, right, rig, frame_size=(600, 800))
    d_lf, d_rf = g.dev(lf), g.dev(rf)
    one = [g.empty((544, 728), torch.uint8) for _ in range(2)]
    pair = [g.empty((544, 728), torch.uint8) for _ in range(2)]
    for side, frame in enumerate((d_lf, d_rf)):
        native.call("nxs_rectify_device", g.ptr(frame), 800, 600, ctypes.byref(cameras[side]),
                    728, 544, g.ptr(one[side]), g.stream())
    native.call("nxs_rectify_pair_device", g.ptr(d_lf), g.ptr(d_rf), 800, 600,
                ctypes.byref(cameras[0]), ctypes.byref(cameras[1]), 728, 544, g.ptr(pair[0]),
                g.ptr(pair[1]), g.stream())
    for a, b in zip(one, pair):
        assert (g.host(a) == g.host(b)).all()


@pytest.mark.parametrize("size", [(64, 48), (97, 31), (9, 7)])
def test_census_pair(native, oracle, size):
    torch = g.torch()
    w, h = size
    left, right = oracle.noise(w, h, 3), oracle.noise(w, h, 4)
    codes = g.empty((2, h, w), torch.int64)
    d_left, d_right = g.dev(left), g.dev(right)  # held until the kernel has read them
    native.call("nxs_census_pair_device", g.ptr(d_left), g.ptr(d_right), w, h,
                g.ptr(codes[0]), g.ptr(codes[1]), g.stream())
    out = g.host(codes).view(np.uint64)
    assert (out[0] == oracle.census(left)).all() and (out[1] == oracle.census(right)).all()


@pytest.mark.parametrize("size,disparities", [((64, 48), 64), ((97, 31), 128), ((3, 5), 16),
                                              ((728, 544), 128), ((4096, 9), 256)])
@pytest.mark.parametrize("stage_mask", [0, 1])
def test_check_median_equals_check_then_median(native, oracle, size, disparities, stage_mask):
    torch = g.torch()
    w, h = size
    rng = np.random.default_rng(w * h)
    # A selection-like disparity and its keys: accepted pixels with winner <= x.
    winner = np.minimum(rng.integers(0, disparities, (h, w)), np.arange(w)[None, :])
    accepted = rng.random((h, w)) < 0.8
    cost = rng.integers(0, 900, (h, w))
    disparity = np.where(accepted, winner + rng.uniform(-0.5, 0.5, (h, w)).astype(np.float32),
                         -1.0).astype(np.float32)
    disparity = np.where(accepted & (disparity < 0), 0.0, disparity).astype(np.float32)
    keys = np.where(accepted, (cost << 16) | winner, 0xFFFFFFFF).astype(np.uint32)
    d_disp, d_keys = g.dev(disparity), g.dev(keys.view(np.int32))
    checked = g.empty((h, w), torch.float32)
    want = g.empty((h, w), torch.float32)
    got = g.empty((h, w), torch.float32)
    native.call("nxs_consistency_device", g.ptr(d_disp), g.ptr(d_keys), w, h, g.ptr(checked),
                g.stream())
    native.call("nxs_median3_device", g.ptr(checked), w, h, stage_mask, g.ptr(want), g.stream())
    native.call("nxs_check_median_device", g.ptr(d_disp), g.ptr(d_keys), w, h, stage_mask,
                g.ptr(got), g.stream())
    assert g.same_bits(g.host(got), g.host(want))
