"""Kernel shapes change no result: the path kernels with 4, 8 or 16 words a
lane (8, 16 or 32 disparities) give bit-identical disparities at every
supported disparity count, odd sizes included, against the oracle; the
batched launch with each path shape agrees with the single-pair matcher."""
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


@pytest.fixture
def words_restored():
    from nx_stereo_b200 import native

    lib = native.load()
    saved = {d: lib.nxs_path_words(d) for d in (64, 96, 128, 192, 256)}
    yield lib
    for d, w in saved.items():
        lib.nxs_set_path_words(d, w)


@pytest.mark.parametrize("disparities", [64, 96, 128, 192, 256])
def test_every_path_shape_matches_the_oracle(ctx, oracle, words_restored, disparities):
    left, right = oracle.scene(161, 53, 9)
    want = oracle.sgm(left, right, disparities, 8)
    want3 = oracle.sgm(left, right, disparities, 3)
    for words in (4, 8, 16):
        assert words_restored.nxs_set_path_words(disparities, words) == 0
        assert words_restored.nxs_path_words(disparities) == words
        assert g.same_bits(ctx.sgm(left, right, disparities=disparities), want), words
        assert g.same_bits(ctx.sgm(left, right, disparities=disparities, paths=3), want3), words


def test_path_shapes_at_728x544(ctx, oracle, words_restored):
    from nx_stereo_b200 import scene

    left, right = scene.rectified_pair(728, 544, seed=31, max_disparity=120)
    want = oracle.fast_sgm(left, right, 128, 8)
    for words in (4, 8, 16):
        words_restored.nxs_set_path_words(128, words)
        assert g.same_bits(ctx.sgm(left, right, disparities=128), want), words


def test_the_refused_shapes(words_restored):
    assert words_restored.nxs_set_path_words(128, 2) != 0
    assert words_restored.nxs_set_path_words(80, 8) != 0


@pytest.mark.parametrize("words", [4, 8, 16])
def test_batched_path_shapes(ctx, words):
    from nx_stereo_b200 import batch, scene

    shapes = [(200, 100, {"disparities": d}) for d in (64, 96, 128, 192, 256)]
    pairs = [scene.rectified_pair(w, h, seed=60 + i, max_disparity=min(56, s["disparities"] - 8))
             for i, (w, h, s) in enumerate(shapes)]
    plan = batch.BatchPlan(ctx, shapes, {"path_words": words})
    for i, (left, right) in enumerate(pairs):
        plan.set_inputs(i, left, right)
    for (w, h, s), (left, right), got in zip(shapes, pairs, plan.run()):
        assert g.same_bits(got, ctx.sgm(left, right, **s)), (words, s)
    plan.close()
