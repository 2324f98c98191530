"""The oracle against the reference itself (CPU).

tests/golden/reference_sgm.npz holds the outputs of the reference's own
shader pipeline for NxStereo.sgm/3 (lib/nx_stereo/vulkan.ex:262-333), run on
the CPU from its GLSL sources by oracle/build_ref.py and
tests/golden/make_reference_fixtures.py. Both of the oracle's formulations
(the literal restatement of lib/nx_stereo.ex:475-683 and the optimised one
of native/stereo_match) must equal them bit for bit: the final disparity of
every case, and at 364x272 also the selection's disparity and winner keys
before the left-right check. Where the shader library itself is present
(built from the reference checkout), fresh seeded cases are compared live.
"""
import os

import numpy as np
import pytest

FIXTURES = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_sgm.npz")
UNIQUENESS = 1.0526315789473684


def load_cases():
    with np.load(FIXTURES) as data:
        names = sorted({k.split("/")[0] for k in data.files})
        return {n: {k.split("/")[1]: data[k] for k in data.files if k.split("/")[0] == n}
                for n in names}


CASES = load_cases()


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def test_the_fixtures_cover_the_reference_settings():
    settings = {tuple(c["settings"][:2]) for c in CASES.values()}
    assert settings == {(64, 3), (64, 8), (128, 3), (128, 8)}
    assert {"scene_364x272_d64_p8", "scene_728x544_d128_p8"} <= set(CASES)


def test_the_reference_outputs_keep_the_reference_tests_assertions():
    # full_range_test.exs:38-54: a texture shifted by 96 columns measures 96 in
    # the interior with both path counts.
    for paths in (3, 8):
        d = CASES[f"shift96_160x24_d128_p{paths}"]["disparity"]
        assert (np.round(d[4:20, 104:152]) == 96).all()


@pytest.mark.parametrize("name", sorted(n for n in CASES if n != "scene_728x544_d128_p8"))
def test_the_oracle_equals_the_reference(oracle, name):
    case = CASES[name]
    d, paths, p1, p2 = (int(v) for v in case["settings"])
    want = bits(case["disparity"])
    got = oracle.sgm(case["left"], case["right"], d, paths, p1, p2, UNIQUENESS)
    assert np.array_equal(bits(got), want)
    fast = oracle.fast_sgm(case["left"], case["right"], d, paths, p1, p2, UNIQUENESS)
    assert np.array_equal(bits(fast), want)


def test_the_fast_oracle_equals_the_reference_at_728x544(oracle):
    case = CASES["scene_728x544_d128_p8"]
    got = oracle.fast_sgm(case["left"], case["right"], 128, 8, 8, 64, UNIQUENESS)
    assert np.array_equal(bits(got), bits(case["disparity"]))
    assert (case["disparity"] > 0).mean() > 0.85


def test_the_oracle_selection_equals_the_reference_before_the_check(oracle):
    case = CASES["scene_364x272_d64_p8"]
    lc, rc = oracle.census(case["left"]), oracle.census(case["right"])
    sums = oracle.aggregate(oracle.costs(lc, rc, 64), 8, 8, 64)
    selected, keys = oracle.select(sums, UNIQUENESS)
    assert np.array_equal(bits(selected), bits(case["selected"]))
    assert np.array_equal(keys, case["keys"])


def _live():
    from oracle import reference_shaders

    if not reference_shaders.available():
        pytest.skip("the reference's shader library is not built here")
    return reference_shaders


@pytest.mark.parametrize("seed", range(6))
def test_fresh_cases_against_the_live_reference(oracle, seed):
    ref = _live()
    rng = np.random.default_rng(1000 + seed)
    w, h = int(rng.integers(9, 140)), int(rng.integers(7, 60))
    d, paths = int(rng.choice([64, 128])), int(rng.choice([3, 8]))
    p2 = int(rng.integers(1, 80))
    p1 = int(rng.integers(0, p2))
    uniqueness = float(rng.uniform(1.0, 1.5))
    if seed % 2:
        left, right = oracle.scene(w, h, seed)
    else:
        left = rng.integers(0, 256, (h, w), dtype=np.uint8)
        right = np.roll(left, int(rng.integers(0, 40)), axis=1)
        right = np.clip(right.astype(int) + rng.integers(-3, 4, (h, w)), 0, 255).astype(np.uint8)
    want = ref.sgm(left, right, d, paths, p1, p2, uniqueness)
    got = oracle.sgm(left, right, d, paths, p1, p2, uniqueness)
    assert np.array_equal(bits(got), bits(want)), (w, h, d, paths, p1, p2, uniqueness)
