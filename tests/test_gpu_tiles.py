"""The path scans' cost stream by bulk tensor copies (the default) against
the per-lane copies: identical path volumes and disparities at every full
lane shape (64, 128 and 256 disparities) over wide, tall, square, odd and
short-lined images, the oracle's disparities beside them, and no copy wait
that ran out of tries."""
import hashlib

import numpy as np
import pytest

from tests import gpu_util as g

pytestmark = pytest.mark.gpu


@pytest.fixture
def lib():
    from nx_stereo_b200 import native

    lib = native.load()
    yield lib
    lib.nxs_set_path_tiles(1)


def path_volumes(lib, left, right, disparities, paths=8, p1=8, p2=64):
    from nx_stereo_b200 import native

    h, w = left.shape
    torch = g.torch()
    span = int(lib.nxs_matcher_span(disparities))
    d_l, d_r = g.dev(left), g.dev(right)
    costs = g.empty((h * w * disparities,), torch.uint8)
    volumes = g.empty((paths * h * w * disparities,), torch.uint8)
    native.call("nxs_census_costs_device_ordered", g.ptr(d_l), g.ptr(d_r), w, h, disparities,
                span, g.ptr(costs), g.stream())
    native.call("nxs_paths_device_ordered", g.ptr(costs), w, h, disparities, paths, p1, p2, span,
                g.ptr(volumes), g.stream())
    return hashlib.sha1(g.host(volumes).tobytes()).hexdigest()


@pytest.mark.parametrize("disparities", [64, 128, 256])
@pytest.mark.parametrize("w,h", [(300, 40), (40, 300), (257, 257), (97, 31), (16, 16), (731, 19)])
def test_tiles_equal_the_per_lane_copies(oracle, lib, disparities, w, h):
    from nx_stereo_b200 import native

    left, right = oracle.scene(w, h, w + h)
    got = {}
    for tiles in (2, 0):
        assert lib.nxs_set_path_tiles(tiles) == 0 and lib.nxs_path_tiles() == tiles
        got[tiles] = path_volumes(lib, left, right, disparities)
    assert got[2] == got[0]
    lib.nxs_set_path_tiles(2)
    ctx = native.Context(0)
    want = oracle.sgm(left, right, disparities, 8)
    assert g.same_bits(ctx.sgm(left, right, disparities=disparities), want)
    assert g.same_bits(ctx.sgm(left, right, disparities=disparities, paths=3),
                       oracle.sgm(left, right, disparities, 3))
    ctx.close()
    assert lib.nxs_path_wait_failures() == 0


def test_tiles_at_the_headline_size(lib):
    from nx_stereo_b200 import scene

    left, right = scene.rectified_pair(728, 544, seed=31, max_disparity=120)
    volumes = {}
    for tiles in (2, 0, 1):
        lib.nxs_set_path_tiles(tiles)
        volumes[tiles] = path_volumes(lib, left, right, 128)
    assert volumes[2] == volumes[0] == volumes[1]
    assert lib.nxs_path_wait_failures() == 0
    assert lib.nxs_set_path_tiles(3) != 0
