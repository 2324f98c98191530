"""The CUDA matcher against the reference itself: every case of
tests/golden/reference_sgm.npz (the reference's own shader pipeline for
NxStereo.sgm/3, lib/nx_stereo/vulkan.ex:262-333, run on the CPU from its
sources) bit for bit, through the single-pair entry point, the no-copy
device entry point and the steps the matcher runs (census+costs, paths,
selection) whose selection must equal the reference's before its check."""
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
