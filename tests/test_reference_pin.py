"""The oracle against the reference itself (CPU).

tests/golden/reference_sgm.npz holds the outputs of the reference's own
shader pipeline for NxStereo.sgm/3 (lib/nx_stereo/vulkan.ex:262-333), run on
the CPU from its GLSL sources by oracle/build_ref.py and
tests/golden/make_reference_fixtures.py. Both of the oracle's formulations
(the literal restatement of lib/nx_stereo.ex:475-683 and the optimised one
of native/stereo_match) must equal them bit for bit: the final disparity of
every case, and at 364x272 also the selection's disparity and winner keys
before the left-right check. tests/golden/reference_stages.npz holds the
stages around the matcher (rectification, despeckle, temporal filter, depth,
point cloud, quality sums) from the reference's shaders: bit for bit but
for rectification, which the reference's own test of its shader holds to one
grey level on at least 99.9% equal pixels (its shader sums the distortion
polynomial left to right, the Nx evaluator and the oracle innermost first),
and the quality sums (1e-5 relative, reduced in another order). Where the
shader library itself is present (built from the reference checkout), fresh
seeded cases are compared live.
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


# ---------------------------------------------------------------- the stages around the matcher
STAGES_FILE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                           "reference_stages.npz")


def load_stages():
    with np.load(STAGES_FILE) as data:
        return {k: data[k] for k in data.files}


STAGES = load_stages()


def camera_of(vector):
    return {"k": vector[:9], "d": vector[9:14], "inverse_pr": vector[14:23]}


def rectified_close(got, want):
    """The reference's own bar for its rectify shader against its Nx code
    (test/nx_stereo/kernels_test.exs:94-96): every pixel within one grey
    level, at least 99.9% of them equal (a sample on a rounding half may
    round the other way)."""
    diff = np.abs(got.astype(int) - want.astype(int))
    return diff.max() <= 1 and (diff == 0).mean() >= 0.999


def test_the_oracle_stages_equal_the_reference(oracle):
    s = STAGES
    h, w = s["left_image"].shape
    for side in ("left", "right"):
        c = camera_of(s[side + "_camera"])
        got = oracle.rectify(s[side + "_frame"], oracle.make_camera(c["k"], c["d"], c["inverse_pr"]),
                             (h, w))
        assert rectified_close(got, s[side + "_image"])
    d = oracle.disparity_stage(s["left_image"], s["right_image"], 64, 8)
    assert np.array_equal(bits(d), bits(s["disparity"]))
    assert np.array_equal(bits(oracle.despeckle(s["disparity"], 12, 1.0, 3)), bits(s["despeckled"]))
    filtered, _, missed = oracle.temporal(s["despeckled"], s["previous"].copy(),
                                          s["missed"].copy(), 0.4, 2.0, 2.0, 255.0)
    assert np.array_equal(bits(filtered), bits(s["filtered"]))
    assert np.array_equal(bits(missed), bits(s["missed_out"]))
    f, baseline, cx, cy = (float(v) for v in s["geometry"])
    mm, m = oracle.depth(s["filtered"], f, baseline)
    assert np.array_equal(mm, s["depth_mm"]) and np.array_equal(bits(m), bits(s["depth_m"]))
    grid, kept = oracle.cloud(s["depth_m"], 4, f, cx, cy, 0.05, 20.0)
    assert kept == int(s["cloud_kept"])
    empty = np.isnan(s["cloud_grid"])
    assert np.array_equal(np.isnan(grid), empty)
    assert np.array_equal(bits(grid[~empty]), bits(s["cloud_grid"][~empty]))
    sums, _ = oracle.quality(s["filtered"], s["previous"].copy())
    assert np.allclose(sums, s["quality_sums"], rtol=1e-5, atol=0)


@pytest.mark.parametrize("w,h", [(728, 544), (1280, 720)])
def test_the_stages_against_the_live_reference_at_the_serving_sizes(oracle, w, h):
    ref = _live()
    from nx_stereo_b200 import scene, segment

    geometry = segment.standard_geometry(w, h)
    left, right = scene.rectified_pair(w, h, seed=5, rectangles=6, max_disparity=56)
    frames = scene.raw_frames(left, right, scene.rig(w, h))
    for side, frame in zip(("left", "right"), frames):
        c = geometry[side + "_camera"]
        want = ref.rectify(frame, c["k"], c["d"], c["inverse_pr"], (h, w))
        got = oracle.rectify(frame, oracle.make_camera(c["k"], c["d"], c["inverse_pr"]), (h, w))
        assert rectified_close(got, want)
    d = oracle.fast_sgm(left, right, 64, 8)
    d = np.where(d > 0, d, np.float32(-1.0)).astype(np.float32)
    assert np.array_equal(bits(oracle.despeckle(d, 12, 1.0, 3)), bits(ref.despeckle(d)))
    f, baseline = geometry["focal_length_px"], geometry["baseline_m"]
    mm, m = oracle.depth(d, f, baseline)
    want_mm, want_m = ref.depth(d, f, baseline)
    assert np.array_equal(mm, want_mm) and np.array_equal(bits(m), bits(want_m))
