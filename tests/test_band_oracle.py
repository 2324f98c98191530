"""The coarse-to-fine oracle against the reference itself (CPU).

tests/golden/reference_band.npz holds the outputs of the reference's own
coarse-to-fine shaders (NxStereo.sgm_band/4 and sgm_coarse_to_fine/3 as
lib/nx_stereo/vulkan.ex:111-255 runs them), made from the reference's GLSL
sources by oracle/build_ref.py and tests/golden/make_reference_fixtures.py.
The oracle (oracle/nxs_oracle_band.c, restated from lib/nx_stereo.ex:138-471)
must equal every case bit for bit, the band bases of the coarse pass too,
and keep the reference tests' own assertions: band_bounds_test.exs (every
match within the right image) and the shrink and band-base definitions.
"""
import os

import numpy as np
import pytest

FIXTURES = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_band.npz")
WINDOW_NAMES = {0: "sparse_9x7", 1: "dense_9x5", 2: "dense_9x5_blend"}


def load_cases():
    with np.load(FIXTURES) as data:
        names = sorted({k.split("/")[0] for k in data.files})
        return {n: {k.split("/")[1]: data[k] for k in data.files if k.split("/")[0] == n}
                for n in names}


CASES = load_cases()


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def run_oracle(oracle, case):
    s = [int(v) for v in case["settings"]]
    band, paths, p1, p2, window = s[:5]
    uniqueness = float(case["uniqueness"])
    if len(s) > 5:  # coarse to fine: coarse paths and margin follow
        return oracle.sgm_coarse_to_fine(case["left"], case["right"], paths, s[5], band, s[6],
                                         WINDOW_NAMES[window], p1, p2, uniqueness, with_base=True)
    return oracle.sgm_band(case["left"], case["right"], case["base"], 128, paths, band,
                           WINDOW_NAMES[window], p1, p2, uniqueness), case["base"]


@pytest.mark.parametrize("name", sorted(CASES))
def test_the_band_oracle_equals_the_reference(oracle, name):
    case = CASES[name]
    got, base = run_oracle(oracle, case)
    assert np.array_equal(base, case["base"])
    assert np.array_equal(bits(got), bits(case["disparity"]))


@pytest.mark.parametrize("name", sorted(n for n in CASES if n.startswith("bounds")))
def test_no_match_leaves_the_right_image(name):
    # band_bounds_test.exs:17-30: -1 or a disparity within 0..min(x, 127).
    d = CASES[name]["disparity"]
    x = np.arange(d.shape[1])[None, :]
    assert (d > 0).any()
    assert ((d == -1.0) | ((d >= 0) & (d <= np.minimum(x, 127)))).all()


def test_shrink_and_band_base_known_answers(oracle):
    image = np.array([[0, 1, 2, 3], [1, 2, 3, 255], [10, 10, 0, 0], [11, 10, 0, 1]], np.uint8)
    # (sum + 2) // 4 of each 2x2 block (lib/nx_stereo.ex:227-238)
    assert oracle.shrink(image).tolist() == [[1, 66], [10, 0]]
    coarse = np.array([[-1.0, 5.25, -1.0], [-1.0, -1.0, -1.0], [-1.0, -1.0, 30.0]], np.float32)
    base = oracle.band_base(coarse, band=16, margin=4)
    # lowest match in each 3x3 neighbourhood, doubled, floored, minus the
    # margin, clipped to 0..112; -1 where the neighbourhood holds none
    want = np.array([[6, 6, 6], [6, 6, 6], [-1, 56, 56]], np.int32)
    assert np.array_equal(base[::2, ::2], want)
    assert np.array_equal(base, np.kron(want, np.ones((2, 2), np.int32)))
    high = oracle.band_base(np.full((2, 2), 63.5, np.float32), band=64, margin=0)
    assert (high == 64).all()  # 127 clipped to 128 - 64


def test_a_full_band_from_zero_is_the_full_search(oracle):
    # sgm_band/4's doc: a band covering every disparity with base 0 gives
    # sgm/3's result; at 64 disparities the band of 64 covers them all.
    left, right = oracle.scene(97, 31, 7)
    base = np.zeros((31, 97), np.int32)
    assert np.array_equal(bits(oracle.sgm_band(left, right, base, 64, 8, 64)),
                          bits(oracle.sgm(left, right, 64, 8)))


def _live():
    from oracle import reference_shaders

    if not reference_shaders.available():
        pytest.skip("the reference's shader library is not built here")
    return reference_shaders


@pytest.mark.parametrize("seed", range(4))
def test_fresh_band_cases_against_the_live_reference(oracle, seed):
    ref = _live()
    rng = np.random.default_rng(500 + seed)
    w, h = int(rng.integers(9, 90)), int(rng.integers(7, 40))
    band = int(rng.choice([8, 16, 32, 64]))
    paths = int(rng.choice([3, 8]))
    census = ["sparse_9x7", "dense_9x5", "dense_9x5_blend"][seed % 3]
    p2 = int(rng.integers(1, 80))
    p1 = int(rng.integers(0, p2))
    left, right = oracle.scene(w, h, seed)
    base = rng.integers(-1, 129 - band, (h, w)).astype(np.int32)
    want = ref.sgm_band(left, right, base, 128, paths, band, census, p1, p2, 1.1)
    got = oracle.sgm_band(left, right, base, 128, paths, band, census, p1, p2, 1.1)
    assert np.array_equal(bits(got), bits(want))
