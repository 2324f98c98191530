"""Parity of the stage kernels (rectification, despeckle, temporal filter,
depth, point cloud, quality) with the oracle, through the C ABI.

Bit-exact: rectified u8 images, despeckled disparity, temporal disparity and
missed counts, depth_mm and depth_m, the cloud grid (NaN positions) and kept
count. Quality sums: within 1e-5 relative, the reference's own tolerance for
reduced sums (test/nx_stereo/native_parity_test.exs:102-110); the kernels
follow the native reduction order, so they are in practice identical.
"""
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


def rectify_gpu(native, frame, cam, size):
    fh, fw = frame.shape
    h, w = size
    d_frame = g.dev(frame)
    d_out = g.empty((h, w), g.torch().uint8)
    c = native.make_camera(cam["k"], cam["d"], cam["inverse_pr"])
    native.call("nxs_rectify_device", g.ptr(d_frame), fw, fh, ctypes.byref(c), w, h,
                g.ptr(d_out), g.stream())
    return g.host(d_out)


@pytest.mark.parametrize("frame_size,size", [((544, 728), (544, 728)), ((544, 728), (272, 364)),
                                             ((480, 640), (300, 500)), ((48, 64), (48, 64))])
def test_rectification_is_bit_exact(native, oracle, frame_size, size):
    from nx_stereo_b200 import rectify, scene

    fh, fw = frame_size
    rig = scene.rig(fw, fh, k1=-0.05, k2=0.01)
    rng = np.random.default_rng(fw)
    frame = rng.integers(0, 256, frame_size).astype(np.uint8)
    for side in ("left", "right"):
        s = rig[side]
        # camera/4 at the working size: scale the calibration as the stage expects.
        cam = rectify.camera(s["k"], [-0.05, 0.01, 0.001, -0.002, 0.0005], s["r"], s["p"])
        want = oracle.rectify(frame, oracle.make_camera(cam["k"], cam["d"], cam["inverse_pr"]),
                              size)
        assert (rectify_gpu(native, frame, cam, size) == want).all()
        moved = rectify.move_rows(cam, 1.5)
        want = oracle.rectify(frame, oracle.make_camera(moved["k"], moved["d"],
                                                        moved["inverse_pr"]), size)
        assert (rectify_gpu(native, frame, moved, size) == want).all()


def test_rectification_identity_known_answers(native, oracle):
    from nx_stereo_b200 import rectify

    k = [100.0, 0.0, 32.0, 0.0, 100.0, 24.0, 0.0, 0.0, 1.0]
    identity = [1.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0, 1.0]
    image = oracle.noise(64, 48, 1)
    cam = rectify.camera(k, [], identity, [100.0, 0, 32.0, 0, 0, 100.0, 24.0, 0, 0, 0, 1.0, 0])
    assert (rectify_gpu(native, image, cam, (48, 64)) == image).all()
    cam = rectify.camera(k, [], identity, [100.0, 0, 35.0, 0, 0, 100.0, 24.0, 0, 0, 0, 1.0, 0])
    shifted = rectify_gpu(native, image, cam, (48, 64))
    assert (shifted[:, 3:] == image[:, :61]).all() and (shifted[:, :3] == 0).all()


def despeckle_gpu(native, disparity, min_support, max_diff, radius=3):
    h, w = disparity.shape
    d_in = g.dev(disparity)
    d_out = g.empty((h, w), g.torch().float32)
    native.call("nxs_despeckle_device", g.ptr(d_in), w, h, float(min_support), float(max_diff),
                radius, g.ptr(d_out), g.stream())
    return g.host(d_out)


def random_disparity(rng, h, w):
    d = rng.uniform(0, 60, (h, w)).astype(np.float32)
    d[rng.random((h, w)) < 0.2] = -1.0
    d[rng.random((h, w)) < 0.05] = 0.0
    # smooth patches so support varies
    d[h // 4:h // 2, w // 4:w // 2] = 20.0 + rng.uniform(-0.6, 0.6, (h // 2 - h // 4, w // 2 - w // 4))
    return d


# Radii 1-5 run the kernel with the radius compiled in, 6-8 the general one.
@pytest.mark.parametrize("radius", [1, 2, 3, 4, 5, 6, 8])
@pytest.mark.parametrize("size", [(97, 131), (33, 1), (1, 40), (128, 64)])
def test_despeckle_is_bit_exact(native, oracle, radius, size):
    rng = np.random.default_rng(radius)
    d = random_disparity(rng, *size)
    for min_support, max_diff in [(12, 1.0), (0, 1.0), (3, 0.25), (24, 8.0)]:
        want = oracle.despeckle(d, min_support, max_diff, radius)
        assert g.same_bits(despeckle_gpu(native, d, min_support, max_diff, radius), want)


def test_despeckle_known_answers(native):
    d = np.full((12, 20), 10.0, np.float32)
    d[:, 15:] = -1.0
    d[5, 17] = 30.0
    got = despeckle_gpu(native, d, 12, 1.0)
    assert got[5, 17] == -1.0 and got[0, 0] == 10.0 and got[5, 5] == 10.0


def test_temporal_is_bit_exact(native, oracle):
    rng = np.random.default_rng(4)
    h, w = 40, 50
    prev = np.full((h, w), -1.0, np.float32)
    missed = np.zeros((h, w), np.float32)
    d_prev, d_missed = g.dev(prev), g.dev(missed)
    for step in range(6):
        cur = random_disparity(rng, h, w)
        want, prev, missed = oracle.temporal(cur, prev, missed, 0.4, 2.0, 2.0, 255.0)
        d_cur = g.dev(cur)
        native.call("nxs_temporal_device", g.ptr(d_cur), g.ptr(d_prev), g.ptr(d_missed), h * w,
                    0.4, 2.0, 2.0, 255.0, g.stream())
        assert g.same_bits(g.host(d_cur), want)
        assert g.same_bits(g.host(d_prev), prev) and g.same_bits(g.host(d_missed), missed)


def test_depth_and_cloud_are_bit_exact(native, oracle):
    rng = np.random.default_rng(5)
    h, w = 136 * 4, 182 * 4
    d = random_disparity(rng, h, w)
    d[0, :5] = [10.0, 0.0, -1.0, 0.0001, 0.36622]
    want_mm, want_m = oracle.depth(d, 873.0, 0.2)
    d_in = g.dev(d)
    d_mm = g.empty((h, w), g.torch().int16)
    d_m = g.empty((h, w), g.torch().float32)
    native.call("nxs_depth_device", g.ptr(d_in), h * w, 873.0, 0.2, g.ptr(d_mm), g.ptr(d_m),
                g.stream())
    assert (g.host(d_mm).view(np.uint16) == want_mm).all()
    assert g.same_bits(g.host(d_m), want_m)
    for decimation in (4, 3, 1):
        want_grid, want_kept = oracle.cloud(want_m, decimation, 873.0, w / 2, h / 2, 0.05, 20.0)
        d_grid = g.empty(want_grid.shape, g.torch().float32)
        d_kept = g.empty((1,), g.torch().int32)
        native.call("nxs_cloud_device", g.ptr(d_m), w, h, decimation, 873.0, w / 2, h / 2, 0.05,
                    20.0, g.ptr(d_grid), g.ptr(d_kept), g.stream())
        grid = g.host(d_grid)
        assert int(g.host(d_kept)[0]) == want_kept
        assert (np.isnan(grid) == np.isnan(want_grid)).all()
        finite = ~np.isnan(want_grid)
        assert g.same_bits(grid[finite], want_grid[finite])


@pytest.mark.parametrize("radius", [1, 3, 5])
@pytest.mark.parametrize("size,decimation", [((182 * 4, 136 * 4), 4), ((97, 131), 3),
                                             ((33, 7), 1), ((4096, 9), 4), ((5, 40), 5)])
def test_despeckle_depth_cloud_in_one_launch(native, oracle, radius, size, decimation):
    """nxs_despeckle_depth_cloud_device equals the oracle's despeckle, then depth on
    its result, then the point cloud of that depth, bit for bit (NaN where no point)."""
    torch = g.torch()
    w, h = size
    rng = np.random.default_rng(w + radius)
    d = random_disparity(rng, h, w)
    d[0, :5] = [10.0, 0.0, -1.0, 0.0001, 0.36622][:min(5, w)]
    speckled = oracle.despeckle(d, 12, 1.0, radius)
    want_mm, want_m = oracle.depth(speckled, 873.0, 0.2)
    want_grid, want_kept = oracle.cloud(want_m, decimation, 873.0, w / 2, h / 2, 0.05, 20.0)
    d_in = g.dev(d)
    out = {"speckled": g.empty((h, w), torch.float32), "mm": g.empty((h, w), torch.int16),
           "m": g.empty((h, w), torch.float32),
           "grid": g.empty(want_grid.shape, torch.float32), "kept": g.empty((1,), torch.int32)}
    out["kept"].fill_(77)  # the launch zeroes the count before adding to it
    native.call("nxs_despeckle_depth_cloud_device", g.ptr(d_in), w, h, 12.0, 1.0, radius, 873.0,
                0.2, decimation, w / 2, h / 2, 0.05, 20.0, g.ptr(out["speckled"]),
                g.ptr(out["mm"]), g.ptr(out["m"]), g.ptr(out["grid"]), g.ptr(out["kept"]),
                g.stream())
    assert g.same_bits(g.host(out["speckled"]), speckled)
    assert (g.host(out["mm"]).view(np.uint16) == want_mm).all()
    assert g.same_bits(g.host(out["m"]), want_m)
    grid = g.host(out["grid"])
    assert int(g.host(out["kept"])[0]) == want_kept
    assert (np.isnan(grid) == np.isnan(want_grid)).all()
    finite = ~np.isnan(want_grid)
    assert g.same_bits(grid[finite], want_grid[finite])
    with pytest.raises(native.NativeError):  # the radii compiled in are 1..5
        native.call("nxs_despeckle_depth_cloud_device", g.ptr(d_in), w, h, 12.0, 1.0, 6, 873.0,
                    0.2, decimation, w / 2, h / 2, 0.05, 20.0, g.ptr(out["speckled"]),
                    g.ptr(out["mm"]), g.ptr(out["m"]), g.ptr(out["grid"]), g.ptr(out["kept"]),
                    g.stream())


def test_quality_sums(native, oracle):
    rng = np.random.default_rng(6)
    h, w = 544, 728
    prev = np.full((h, w), -1.0, np.float32)
    d_prev = g.dev(prev)
    for step in range(3):
        cur = random_disparity(rng, h, w)
        want, prev = oracle.quality(cur, prev)
        d_cur = g.dev(cur)
        d_sums = g.empty((5,), g.torch().float32)
        native.call("nxs_quality_device", g.ptr(d_cur), g.ptr(d_prev), w, h, g.ptr(d_sums),
                    g.stream())
        got = g.host(d_sums)
        assert np.allclose(got, want, rtol=1e-5, atol=0)
        assert g.same_bits(g.host(d_prev), prev)
