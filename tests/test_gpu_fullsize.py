"""The matcher at the benchmark sizes: bit-exact against the oracle's optimised
formulation at 728x544 with 128 disparities (8 and 3 paths) and at 1920x1080
with 256 disparities, and size-independent properties at full size: a
texture shifted by s columns measures s, unrelated images at a uniqueness of
1000 match nowhere, and identical images (disparity 0 everywhere) are
unmatched after Stage.Disparity's mask."""
import numpy as np
import pytest

from tests import gpu_util as g

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from nx_stereo_b200 import native

    c = native.Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("paths", [8, 3])
def test_728x544_128_disparities_bit_exact(ctx, oracle, paths):
    from nx_stereo_b200 import scene

    left, right = scene.rectified_pair(728, 544, seed=11, rectangles=6, max_disparity=120)
    want = oracle.fast_sgm(left, right, 128, paths)
    assert g.same_bits(ctx.sgm(left, right, disparities=128, paths=paths), want)


@pytest.mark.parametrize("w,h,d", [(640, 480, 96), (1280, 720, 192)])
def test_batched_workload_shapes_beyond_the_reference_bit_exact(ctx, oracle, w, h, d):
    # Two of the batched workload's full-size shapes at disparity counts the
    # reference refuses (96 and 192), single pairs against the oracle.
    from nx_stereo_b200 import scene

    left, right = scene.rectified_pair(w, h, seed=w + d, rectangles=6, max_disparity=d - 8)
    want = oracle.fast_sgm(left, right, d, 8)
    got = ctx.sgm(left, right, disparities=d, paths=8)
    assert g.same_bits(got, want)
    assert (got > 0).mean() > 0.5


def test_1920x1080_256_disparities_bit_exact(ctx, oracle):
    from nx_stereo_b200 import scene

    left, right = scene.rectified_pair(1920, 1080, seed=12, rectangles=12, min_disparity=8,
                                       max_disparity=240, sigma=3.0)
    want = oracle.fast_sgm(left, right, 256, 8)
    got = ctx.sgm(left, right, disparities=256, paths=8)
    assert g.same_bits(got, want)
    assert (got > 0).mean() > 0.5


def test_a_shifted_texture_measures_its_shift_at_full_size(ctx, oracle):
    shift = 100
    texture = oracle.noise(1920 + shift, 1080, 21)
    left, right = texture[:, :1920], texture[:, shift:shift + 1920]
    d = ctx.sgm(np.ascontiguousarray(left), np.ascontiguousarray(right), disparities=256)
    interior = d[8:-8, 260:-8]
    # Every winner is the shift; on 1.76 million noise pixels a few parabola
    # corrections reach 0.1 (the oracle gives the same 1183).
    assert (np.abs(interior - shift) < 0.5).all()
    assert (np.abs(interior - shift) < 0.1).mean() > 0.999


def test_unrelated_and_identical_images_at_full_size(ctx, oracle):
    left, right = oracle.noise(728, 544, 5), oracle.noise(728, 544, 6)
    assert (ctx.sgm(left, right, disparities=128, uniqueness=1000.0) == -1.0).all()
    assert (ctx.sgm(left, left, disparities=128, stage_mask=True) == -1.0).all()
