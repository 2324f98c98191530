"""The CUDA matcher against the reference itself: every case of
tests/golden/reference_sgm.npz (the reference's own shader pipeline for
NxStereo.sgm/3, lib/nx_stereo/vulkan.ex:262-333, run on the CPU from its
sources) bit for bit, through the single-pair entry point, the no-copy
device entry point and the steps the matcher runs (census+costs, paths,
selection) whose selection must equal the reference's before its check; and
the stage kernels against tests/golden/reference_stages.npz."""
import numpy as np
import pytest

from tests import gpu_util as g
from tests.test_reference_pin import CASES, UNIQUENESS, bits

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from nx_stereo_b200 import native

    c = native.Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("name", sorted(CASES))
def test_the_cuda_matcher_equals_the_reference(ctx, name):
    case = CASES[name]
    d, paths, p1, p2 = (int(v) for v in case["settings"])
    got = ctx.sgm(case["left"], case["right"], disparities=d, paths=paths, p1=p1, p2=p2,
                  uniqueness=UNIQUENESS)
    assert np.array_equal(bits(got), bits(case["disparity"]))


@pytest.mark.parametrize("name", ["scene_364x272_d64_p8", "scene_728x544_d128_p8"])
def test_the_device_entry_point_equals_the_reference(ctx, name):
    case = CASES[name]
    h, w = case["left"].shape
    d, paths = int(case["settings"][0]), int(case["settings"][1])
    d_left, d_right = g.dev(case["left"]), g.dev(case["right"])
    out = g.empty((h, w), g.torch().float32)
    ctx.sgm_device(g.ptr(d_left), g.ptr(d_right), w, h, g.ptr(out), stream=g.stream(),
                   disparities=d, paths=paths)
    assert np.array_equal(bits(g.host(out)), bits(case["disparity"]))


def test_the_cuda_selection_equals_the_reference_before_the_check():
    from nx_stereo_b200 import native

    case = CASES["scene_364x272_d64_p8"]
    h, w = case["left"].shape
    torch = g.torch()
    span = native.load().nxs_matcher_span(64)
    d_left, d_right = g.dev(case["left"]), g.dev(case["right"])
    costs = g.empty((h, w, 64), torch.uint8)
    paths = g.empty((8, h, w, 64), torch.uint8)
    selected = g.empty((h, w), torch.float32)
    keys = g.empty((h, w), torch.int32)
    native.call("nxs_census_costs_device_ordered", g.ptr(d_left), g.ptr(d_right), w, h, 64, span,
                g.ptr(costs), g.stream())
    native.call("nxs_paths_device_ordered", g.ptr(costs), w, h, 64, 8, 8, 64, span, g.ptr(paths),
                g.stream())
    native.call("nxs_select_paths_device_ordered", g.ptr(paths), w, h, 64, 8,
                UNIQUENESS, span, g.ptr(selected), g.ptr(keys), g.stream())
    assert np.array_equal(bits(g.host(selected)), bits(case["selected"]))
    assert np.array_equal(g.host(keys).view(np.uint32), case["keys"])


def test_the_cuda_stages_equal_the_reference():
    """Rectification of both raw frames, the matcher with Stage.Disparity's
    mask, despeckle, a temporal step, depth, the point cloud and the quality
    sums, each on the reference's own input for it, against the reference's
    shaders (tests/golden/reference_stages.npz)."""
    import ctypes

    from nx_stereo_b200 import native
    from tests.test_reference_pin import STAGES as s
    from tests.test_reference_pin import camera_of, rectified_close

    torch = g.torch()
    native.load()
    h, w = s["left_image"].shape
    for side in ("left", "right"):
        frame, c = s[side + "_frame"], camera_of(s[side + "_camera"])
        fh, fw = frame.shape
        d_frame, d_out = g.dev(frame), g.empty((h, w), torch.uint8)
        cam = native.make_camera(c["k"], c["d"], c["inverse_pr"])
        native.call("nxs_rectify_device", g.ptr(d_frame), fw, fh, ctypes.byref(cam), w, h,
                    g.ptr(d_out), g.stream())
        assert rectified_close(g.host(d_out), s[side + "_image"])
    ctx = native.Context(0)
    d = ctx.sgm(s["left_image"], s["right_image"], disparities=64, paths=8, stage_mask=True)
    ctx.close()
    assert np.array_equal(bits(d), bits(s["disparity"]))
    d_in, d_out = g.dev(s["disparity"]), g.empty((h, w), torch.float32)
    native.call("nxs_despeckle_device", g.ptr(d_in), w, h, 12.0, 1.0, 3, g.ptr(d_out), g.stream())
    assert np.array_equal(bits(g.host(d_out)), bits(s["despeckled"]))
    d_cur, d_prev, d_missed = g.dev(s["despeckled"]), g.dev(s["previous"]), g.dev(s["missed"])
    native.call("nxs_temporal_device", g.ptr(d_cur), g.ptr(d_prev), g.ptr(d_missed), h * w, 0.4,
                2.0, 2.0, 255.0, g.stream())
    assert np.array_equal(bits(g.host(d_cur)), bits(s["filtered"]))
    assert np.array_equal(bits(g.host(d_missed)), bits(s["missed_out"]))
    f, baseline, cx, cy = (float(v) for v in s["geometry"])
    d_filtered = g.dev(s["filtered"])
    d_mm, d_m = g.empty((h, w), torch.int16), g.empty((h, w), torch.float32)
    native.call("nxs_depth_device", g.ptr(d_filtered), h * w, f, baseline, g.ptr(d_mm),
                g.ptr(d_m), g.stream())
    assert np.array_equal(g.host(d_mm).view(np.uint16), s["depth_mm"])
    assert np.array_equal(bits(g.host(d_m)), bits(s["depth_m"]))
    d_grid = g.empty(s["cloud_grid"].shape, torch.float32)
    d_kept = g.empty((1,), torch.int32)
    native.call("nxs_cloud_device", g.ptr(d_m), w, h, 4, f, cx, cy, 0.05, 20.0, g.ptr(d_grid),
                g.ptr(d_kept), g.stream())
    grid, empty = g.host(d_grid), np.isnan(s["cloud_grid"])
    assert int(g.host(d_kept)[0]) == int(s["cloud_kept"])
    assert np.array_equal(np.isnan(grid), empty)
    assert np.array_equal(bits(grid[~empty]), bits(s["cloud_grid"][~empty]))
    d_prev = g.dev(s["previous"])
    d_sums = g.empty((5,), torch.float32)
    native.call("nxs_quality_device", g.ptr(d_filtered), g.ptr(d_prev), w, h, g.ptr(d_sums),
                g.stream())
    assert np.allclose(g.host(d_sums), s["quality_sums"], rtol=1e-5, atol=0)
