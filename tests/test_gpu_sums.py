"""The summing path scan (every direction adds its path costs into one u16
aggregate volume with f16x2 reductions on the integer bit patterns, then
selection reads that one volume) gives the same disparities as the path
volumes and as the oracle: every disparity count, 8 and 3 paths, odd sizes,
the penalties at their limits (the largest sums, 8 x 127), and the
headline size; the mode knob."""
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
def lib():
    from nx_stereo_b200 import native

    lib = native.load()
    yield lib
    lib.nxs_set_path_sums(0)


@pytest.mark.parametrize("disparities", [64, 96, 128, 192, 256])
def test_summing_equals_the_oracle_and_the_path_volumes(ctx, oracle, lib, disparities):
    for w, h, seed in ((161, 53, 9), (300, 17, 2), (37, 129, 4)):
        left, right = oracle.scene(w, h, seed)
        for paths in (8, 3):
            want = oracle.sgm(left, right, disparities, paths)
            results = []
            for mode in (1, 0):
                assert lib.nxs_set_path_sums(mode) == 0
                assert lib.nxs_path_sums(w, h, disparities) == (1 if mode else 0)
                results.append(ctx.sgm(left, right, disparities=disparities, paths=paths))
            assert g.same_bits(results[0], want), (w, h, paths)
            assert g.same_bits(results[1], want), (w, h, paths)


@pytest.mark.parametrize("p1,p2", [(0, 79), (78, 79), (0, 1), (10, 40)])
def test_summing_at_the_penalty_limits(ctx, oracle, lib, p1, p2):
    # p2 79 with costs up to 48 gives path costs up to 127, sums up to 1016.
    rng = np.random.default_rng(p1 * 100 + p2)
    left = rng.integers(0, 256, (47, 211), dtype=np.uint8)
    right = rng.integers(0, 256, (47, 211), dtype=np.uint8)  # unrelated: high costs everywhere
    lib.nxs_set_path_sums(1)
    for disparities in (64, 128):
        want = oracle.sgm(left, right, disparities, 8, p1, p2)
        got = ctx.sgm(left, right, disparities=disparities, p1=p1, p2=p2)
        assert g.same_bits(got, want), disparities


def test_summing_at_728x544(ctx, oracle, lib):
    from nx_stereo_b200 import scene

    left, right = scene.rectified_pair(728, 544, seed=31, max_disparity=120)
    want = oracle.fast_sgm(left, right, 128, 8)
    lib.nxs_set_path_sums(1)
    assert g.same_bits(ctx.sgm(left, right, disparities=128), want)
    assert g.same_bits(ctx.sgm(left, right, disparities=128, stage_mask=True),
                       np.where(want > 0, want, np.float32(-1.0)).astype(np.float32))


def test_the_mode_knob(lib):
    assert lib.nxs_set_path_sums(2) != 0
    assert lib.nxs_set_path_sums(0) == 0 and lib.nxs_path_sums(728, 544, 128) == 0
    assert lib.nxs_set_path_sums(1) == 0 and lib.nxs_path_sums(728, 544, 128) == 1
    lib.nxs_set_path_words(128, 4)
    assert lib.nxs_path_sums(728, 544, 128) == 0  # the aggregate layout has 8 words a lane
    lib.nxs_set_path_words(128, 8)
