"""Pins the CPU oracle to the reference's own known-answer tests.

The reference ships no stored golden vectors, so the oracle is pinned by
restating the assertions of its unit and integration tests (Rust
native/stereo_match/src/*.rs test modules, Elixir test/nx_stereo/*.exs) on the
same inputs, and by the reference's differential check: the optimised
formulation equals the step-by-step one bit for bit (lib.rs:535-628).
"""
import numpy as np
import pytest


def same_bits(a, b):
    a, b = np.asarray(a, np.float32), np.asarray(b, np.float32)
    return a.shape == b.shape and bool((a.view(np.uint32) == b.view(np.uint32)).all())


# ---------------------------------------------------------------- census
def test_census_bits_follow_the_neighbour_order(oracle):
    # census.rs:122-151: one pixel two levels darker, two rows up and three
    # columns right of the centre, sets bit 8 + 6.
    image = np.full((7, 9), 100, np.uint8)
    image[1, 7] = 98
    assert int(oracle.census(image)[3, 4]) == 1 << 14
    image = np.full((7, 9), 100, np.uint8)
    image[3, 4] = 102
    assert int(oracle.census(image)[3, 4]) == (1 << 48) - 1, "every neighbour two levels below"
    image[3, 4] = 101
    assert int(oracle.census(image)[3, 4]) == 0, "one level below does not count"


def test_costs_are_hamming_distances_with_zero_codes_past_the_edge(oracle):
    left, right = oracle.noise(70, 9, 1), oracle.noise(70, 9, 2)
    lc, rc = oracle.census(left), oracle.census(right)
    costs = oracle.costs(lc, rc, 64)
    y, x = 4, 30
    for d in (0, 1, 30, 31, 63):
        feature = int(rc[y, x - d]) if x >= d else 0
        assert costs[y, x, d] == bin(int(lc[y, x]) ^ feature).count("1")
    assert costs.max() <= 48


# ---------------------------------------------------------------- paths
def test_path_values_stay_within_p2_plus_48(oracle):
    # paths.rs:424-452: at the extreme penalties every path cost is <= p2 + 48.
    rng = np.random.default_rng(9)
    for p1, p2 in [(0, 1), (8, 64), (78, 79)]:
        costs = rng.integers(0, 49, size=(23, 17, 64)).astype(np.int32)
        for direction in [(0, 1), (1, 0), (1, 1), (-1, -1)]:
            path = oracle.path(costs, direction, p1, p2)
            assert path.max() <= p2 + 48
            assert path.min() >= 0


def test_path_starts_from_zero_where_it_enters(oracle):
    costs = np.arange(5 * 4 * 64, dtype=np.int32).reshape(5, 4, 64) % 49
    for direction, edge in [((0, 1), (slice(None), 0)), ((0, -1), (slice(None), 3)),
                            ((1, 0), (0, slice(None))), ((-1, 0), (4, slice(None)))]:
        path = oracle.path(costs, direction, 8, 64)
        assert (path[edge] == costs[edge]).all()


# ---------------------------------------------------------------- select
def test_select_ties_go_to_the_lower_disparity_and_the_edge_is_respected(oracle):
    # select.rs:247-261
    def winner(sums, x):
        volume = np.zeros((1, x + 1, 64), np.int32)
        volume[0, x] = sums
        return int(oracle.select(volume, 1.0)[1][0, x]) & 0xFFFF

    sums = np.full(64, 100, np.int32)
    sums[10] = sums[11] = 5
    assert winner(sums, 63) == 10
    sums[3] = 1
    assert winner(sums, 63) == 3
    sums[0] = 50
    assert winner(sums, 2) == 0, "disparities past x lose"


def test_select_refines_with_the_parabola_and_keys_hold_cost_and_winner(oracle):
    volume = np.full((1, 40, 64), 500, np.int32)
    volume[0, 30, 9:12] = [110, 100, 130]
    disparity, keys = oracle.select(volume, 1.0526316)
    correction = np.float32(110 - 130) / (np.float32(2) * np.float32(110 + 130 - 200))
    assert disparity[0, 30] == np.float32(10) + correction
    assert int(keys[0, 30]) == (100 << 16) | 10


# ---------------------------------------------------------------- check
def test_a_tie_on_a_right_pixel_favours_the_larger_disparity(oracle):
    # check.rs:395-407
    keys = np.full((1, 16), 0xFFFFFFFF, np.uint32)
    keys[0, 10] = (3 << 16) | 5
    keys[0, 12] = (3 << 16) | 7
    disparity = np.full((1, 16), -1.0, np.float32)
    disparity[0, 10], disparity[0, 12] = 5.0, 7.0
    out = oracle.consistency(disparity, keys, 64)
    assert (out[0, 10], out[0, 12]) == (-1.0, 7.0)


def test_median_is_the_sorted_middle_with_replicated_borders(oracle):
    rng = np.random.default_rng(5)
    image = (rng.integers(0, 9, size=(7, 13)) - 1).astype(np.float32)
    got = oracle.median3(image)
    padded = np.pad(image, 1, mode="edge")
    for y in range(7):
        for x in range(13):
            assert got[y, x] == np.sort(padded[y:y + 3, x:x + 3].ravel())[4]


# ---------------------------------------------------------------- the matcher
CASES = [((64, 48), 64, 3), ((64, 48), 64, 8), ((64, 48), 128, 3), ((64, 48), 128, 8),
         ((97, 31), 64, 3), ((97, 31), 64, 8), ((97, 31), 128, 3), ((97, 31), 128, 8)]


@pytest.mark.parametrize("size,disparities,paths", CASES)
def test_the_optimised_formulation_equals_the_step_by_step_one(oracle, size, disparities, paths):
    # lib.rs:535-568: scenes and noise, bit for bit.
    w, h = size
    left, right = oracle.scene(w, h, 7)
    assert same_bits(oracle.fast_sgm(left, right, disparities, paths),
                     oracle.sgm(left, right, disparities, paths))
    left, right = oracle.noise(w, h, 1), oracle.noise(w, h, 2)
    assert same_bits(oracle.fast_sgm(left, right, disparities, paths),
                     oracle.sgm(left, right, disparities, paths))


@pytest.mark.parametrize("p1,p2,uniqueness", [(0, 1, 1.0), (4, 40, 1.2), (78, 79, 2.5),
                                              (10, 79, 1.0526316)])
def test_other_penalties_and_uniqueness(oracle, p1, p2, uniqueness):
    # lib.rs:570-593
    left, right = oracle.scene(80, 40, 3)
    for paths in (3, 8):
        assert same_bits(oracle.fast_sgm(left, right, 64, paths, p1, p2, uniqueness),
                         oracle.sgm(left, right, 64, paths, p1, p2, uniqueness))


def test_a_shifted_scene_measures_its_disparity(oracle):
    # lib.rs:630-644
    w, h = 96, 64
    left, right = oracle.scene(w, h, 11)
    disparity = oracle.sgm(left, right, 64, 8)
    x, y = 60, 20
    u = (x - 4.0 - 6.0 * y / h) / (1.0 + 30.0 / w)
    assert abs(disparity[y, x] - (x - u)) < 1.0


def test_recovers_the_disparity_of_a_shifted_texture(oracle):
    # nx_stereo_test.exs:58-66 with the xorshift texture standing in for :rand.
    texture = oracle.noise(96 + 5, 24, 1)
    left, right = texture[:, :96], texture[:, 5:101]
    disparity = oracle.sgm(left, right)
    interior = disparity[4:24 - 4, 70:96 - 4]
    assert (np.abs(interior - 5.0) < 0.1).all()


def test_marks_pixels_without_a_reliable_match(oracle):
    # nx_stereo_test.exs:68-75: unrelated images at uniqueness 1000.
    left, right = oracle.noise(80, 16, 1), oracle.noise(80, 16, 2)
    assert (oracle.sgm(left, right, uniqueness=1000.0) == -1.0).all()


def test_the_stage_masks_disparity_zero(oracle):
    # segment.rs:641-678 / disparity.ex:162: a pair matched at disparity 0 is unmatched.
    image = oracle.noise(64, 48, 4)
    stage = oracle.disparity_stage(image, image)
    raw = oracle.sgm(image, image)
    assert (raw[raw >= 0] == 0).mean() > 0.9
    assert ((stage == -1.0) | (stage > 0)).all()
    assert (stage[raw <= 0] == -1.0).all()


# ---------------------------------------------------------------- filters
def test_despeckle_drops_islands_and_keeps_surfaces(oracle):
    # filters.rs:571-586
    d = np.full((12, 20), 10.0, np.float32)
    d[:, 15:] = -1.0
    d[5, 17] = 30.0
    got = oracle.despeckle(d, 12, 1.0, 3)
    assert got[5, 17] == -1.0 and got[0, 0] == 10.0 and got[5, 5] == 10.0
    assert (got[5, 15:] == -1.0).all()


def test_despeckle_reads_a_disparity_of_0_as_unmatched(oracle):
    d = np.zeros((10, 12), np.float32)
    d[5, 5] = 0.5
    assert (oracle.despeckle(d, 12, 1.0, 3) == -1.0).all()


def test_despeckle_counts_the_neighbours_within_its_radius(oracle):
    d = np.full((5, 5), 10.0, np.float32)
    assert oracle.despeckle(d, 9, 0.0, 1)[2, 2] == -1.0
    assert oracle.despeckle(d, 8, 0.0, 1)[2, 2] == 10.0
    assert oracle.despeckle(d, 24, 0.0, 3)[2, 2] == 10.0


def test_despeckle_elixir_cases(oracle):
    # filter_test.exs:6-45
    s = np.full((12, 12), 10.0, np.float32)
    s[:, 8:12] = -1.0
    s[5, 3] = 30.0
    s[6, 10] = 12.0
    f = oracle.despeckle(s, 12, 1.0)
    assert f[5, 3] == -1.0 and f[6, 10] == -1.0 and f[0, 0] == 10.0 and f[11, 7] == 10.0
    assert f[0, 9] == -1.0
    assert same_bits(oracle.despeckle(s, 0, 1.0), s)
    image = np.full((9, 9), -1.0, np.float32)
    image[3:6, 3:6] = 29.5
    image[4, 4] = 30.0
    assert oracle.despeckle(image, 8, 1.0)[4, 4] == 30.0
    assert oracle.despeckle(image, 9, 1.0)[4, 4] == -1.0
    assert oracle.despeckle(image, 1, 0.25)[4, 4] == -1.0
    assert oracle.despeckle(image, 8, 1.0, 1)[4, 4] == 30.0


def test_temporal_known_answers(oracle):
    # filters.rs:616-670
    out, prev, miss = oracle.temporal([10.0, 0.0], [-1.0, -1.0], [0.0, 0.0], 0.4, 2.0, 1.0)
    out, prev, miss = oracle.temporal([0.0, 1.0], prev, miss, 0.4, 2.0, 1.0)
    assert out.tolist() == [10.0, 1.0]
    prev, miss = np.full(3, -1.0, np.float32), np.zeros(3, np.float32)
    seq = [[10.0, 10.0, 10.0], [11.0, 20.0, -1.0], [11.0, 20.0, -1.0]]
    want = [[10.0, 10.0, 10.0], [10.5, 20.0, 10.0], [10.75, 20.0, -1.0]]
    for cur, expected in zip(seq, want):
        out, prev, miss = oracle.temporal(cur, prev, miss, 0.5, 2.0, 1.0)
        assert out.tolist() == expected

    def held(max_missed):
        out, prev, miss = oracle.temporal([10.0], [-1.0], [0.0], 1.0, 2.0, 2.0, max_missed)
        values = []
        for _ in range(4):
            out, prev, miss = oracle.temporal([-1.0], prev, miss, 1.0, 2.0, 2.0, max_missed)
            values.append(float(out[0]))
        return values

    assert held(255.0) == [10.0, 10.0, -1.0, -1.0]
    assert held(1.0) == [10.0, 10.0, 10.0, 10.0]
    # filter_test.exs:69-90
    out, _, miss = oracle.temporal([12.0, 20.0, 5.0, -1.0], [10.0, 10.0, -1.0, -1.0],
                                   [0, 0, 3, 0], 0.5, 2.0, 0.0)
    assert out.tolist() == [11.0, 20.0, 5.0, -1.0] and miss.tolist() == [0.0, 0.0, 0.0, 1.0]
    out, _, miss = oracle.temporal([-1.0], [8.0], [1.0], 0.4, 2.0, 2.0)
    assert (out.tolist(), miss.tolist()) == ([8.0], [2.0])
    out, _, miss = oracle.temporal([-1.0], [8.0], [2.0], 0.4, 2.0, 2.0)
    assert (out.tolist(), miss.tolist()) == ([-1.0], [3.0])
    out, _, miss = oracle.temporal([-1.0], [-1.0], [255.0], 0.4, 2.0, 2.0)
    assert (out.tolist(), miss.tolist()) == ([-1.0], [255.0])


# ---------------------------------------------------------------- depth, cloud, quality
def test_depth_known_answers(oracle):
    # depth.rs:95-107, depth_test.exs:6-28
    mm, m = oracle.depth(np.array([10.0, 0.0, -1.0, 1.0e-4], np.float32), 100.0, 0.1)
    assert m[:3].tolist() == [1.0, 0.0, 0.0] and mm.tolist() == [1000, 0, 0, 0]
    mm, _ = oracle.depth(np.array([1.0, 0.9999], np.float32), 65535.0, 0.001)
    assert mm.tolist() == [65535, 0]
    mm, m = oracle.depth(np.array([[10.0, 0.0, -1.0, 0.0001, 0.36622]], np.float32), 400.0, 0.06)
    assert mm.tolist() == [[2400, 0, 0, 0, 65534]]
    assert abs(m[0, 0] - 2.4) < 1e-6 and abs(m[0, 3] - 240000.0) < 1.0
    mm, _ = oracle.depth(np.array([[10.0, 20.0]], np.float32), 400.0, -0.06)
    assert mm.tolist() == [[0, 0]]


def test_cloud_known_answers(oracle):
    # depth.rs:109-154, depth_test.exs:30-86
    depth_m = np.array([2.0, 9.0, 30.0, 9.0, 9.0, 9.0, 0.0, 9.0], np.float32).reshape(2, 4)
    grid, kept = oracle.cloud(depth_m, 2, 2.0, 1.0, 0.0, 0.05, 20.0)
    assert kept == 1 and grid.ravel()[:3].tolist() == [-1.0, 0.0, 2.0]
    assert np.isnan(grid.ravel()[3:]).all()
    depth_m = (1.0 + np.arange(8 * 11) // 8).astype(np.float32).reshape(11, 8)
    grid, kept = oracle.cloud(depth_m, 4, 2.0, 0.0, 0.0, 0.05, 20.0)
    assert kept == 4 and grid.ravel()[6:12].tolist() == [0.0, 10.0, 5.0, 10.0, 10.0, 5.0]
    depth_m = np.array([[0.5, 1.0, 1.5, 2.5, 3.0, 3.5]], np.float32)
    grid, kept = oracle.cloud(depth_m, 1, 1.0, 0.0, 0.0, 1.0, 3.0)
    z = grid[0, :, 2]
    assert kept == 2 and z[2] == 1.5 and z[3] == 2.5 and np.isnan(z[[0, 1, 4, 5]]).all()
    grid, kept = oracle.cloud(np.full((48, 64), 2.0, np.float32), 4, 100.0, 32.0, 24.0)
    assert grid.shape == (12, 16, 3) and kept == 192
    assert abs(grid[1, 1, 0] - (4 - 32) * 2.0 / 100) < 1e-6
    assert abs(grid[1, 1, 1] - (4 - 24) * 2.0 / 100) < 1e-6 and grid[1, 1, 2] == 2.0
    depth_m = (np.arange(270, dtype=np.float32)[:, None] + np.zeros((1, 8), np.float32)) + 1.0
    grid, _ = oracle.cloud(depth_m, 4, 100.0, 0.0, 0.0, 0.05, 1000.0)
    assert grid.shape == (67, 2, 3)
    assert [int(v - 1) for v in grid[:, 0, 2]] == [v * 4 for v in range(67)]
    grid, kept = oracle.cloud(np.array([[0.0, 0.04, 0.06, 19.0, 21.0, 5.0]], np.float32), 1,
                              100.0, 0.0, 0.0, 0.05, 20.0)
    assert np.isnan(grid[0, :, 2]).astype(int).tolist() == [1, 1, 0, 0, 1, 0] and kept == 3


def test_quality_counts_matched_pixels_and_their_change(oracle):
    # measures.rs:396-407
    prev = np.full((2, 2), -1.0, np.float32)
    sums, prev = oracle.quality(np.array([[2.0, 0.0], [-1.0, 4.0]], np.float32), prev)
    assert sums.tolist() == [2.0, 6.0, 20.0, 0.0, 0.0]
    sums, prev = oracle.quality(np.array([[3.0, 1.0], [1.0, 4.0]], np.float32), prev)
    assert sums.tolist() == [4.0, 9.0, 27.0, 2.0, 1.0]


# ---------------------------------------------------------------- rectification
def _identity_camera(oracle, width, height):
    cx, cy = width / 2.0, height / 2.0
    return oracle.make_camera([100.0, 0.0, cx, 0.0, 100.0, cy, 0.0, 0.0, 1.0], [0.0] * 5,
                              [0.01, 0.0, -cx / 100.0, 0.0, 0.01, -cy / 100.0, 0.0, 0.0, 1.0])


def test_an_identity_camera_copies_the_frame(oracle):
    # rectify.rs:173-188
    w, h = 16, 8
    frame = (np.arange(w * h) * 7 % 256).astype(np.uint8).reshape(h, w)
    assert (oracle.rectify(frame, _identity_camera(oracle, w, h), (h, w)) == frame).all()


def test_halving_the_size_averages_each_square_of_four(oracle):
    # rectify.rs:190-211
    w, h = 8, 4
    frame = (np.arange(4 * w * h) % 2 * 100).astype(np.uint8).reshape(2 * h, 2 * w)
    out = oracle.rectify(frame, _identity_camera(oracle, w, h), (h, w))
    assert out[1, 1] == 50


def _camera64(oracle, d, fx, cx, cy):
    # Rectify.camera/4 for K = [[100,0,32],[0,100,24],[0,0,1]], R = I and
    # P = [[fx,0,cx,0],[0,fx,cy,0],[0,0,1,0]], built in f64 then cast.
    p3 = np.array([[fx, 0.0, cx], [0.0, fx, cy], [0.0, 0.0, 1.0]])
    return oracle.make_camera([100.0, 0.0, 32.0, 0.0, 100.0, 24.0, 0.0, 0.0, 1.0],
                              (list(d) + [0.0] * 5)[:5], np.linalg.inv(p3).ravel())


def test_identity_calibration_and_a_principal_point_shift(oracle):
    # rectify_test.exs:38-56
    image = oracle.noise(64, 48, 1)
    assert (oracle.rectify(image, _camera64(oracle, [], 100.0, 32.0, 24.0), (48, 64)) == image).all()
    shifted = oracle.rectify(image, _camera64(oracle, [], 100.0, 35.0, 24.0), (48, 64))
    assert (shifted[:, 3:64] == image[:, 0:61]).all() and (shifted[:, 0:3] == 0).all()


def test_radial_distortion_maps_a_pixel_where_the_formula_says(oracle):
    # rectify_test.exs:58-87
    k1, u, v = 0.5, 60, 40
    x, y = (u - 32) / 100, (v - 24) / 100
    radial = 1 + k1 * (x * x + y * y)
    sx, sy = 100 * x * radial + 32, 100 * y * radial + 24
    image = np.zeros((48, 64), np.uint8)
    image[int(np.floor(sy)):int(np.floor(sy)) + 2, int(np.floor(sx)):int(np.floor(sx)) + 2] = 255
    out = oracle.rectify(image, _camera64(oracle, [k1], 100.0, 32.0, 24.0), (48, 64))
    assert out[v, u] == 255
    out = oracle.rectify(image, _camera64(oracle, [], 100.0, 32.0, 24.0), (48, 64))
    assert out[v, u] == 0
