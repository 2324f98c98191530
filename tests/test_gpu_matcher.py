"""Parity of the CUDA matcher with the oracle, through the C ABI.

Integer outputs (census codes, costs, aggregated costs, integer disparity and
keys) must be bit-exact; the f32 subpixel disparity keeps the reference's
operation order and must be identical bit for bit (tolerance 0).
"""
import numpy as np
import pytest

from tests import gpu_util as g

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def native():
    from nx_stereo_b200 import native as n

    n.load()
    return n


@pytest.fixture(scope="module")
def ctx(native):
    c = native.Context(0)
    yield c
    c.close()


def census_gpu(native, image):
    h, w = image.shape
    d_image = g.dev(image)
    d_codes = g.empty((h, w), g.torch().int64)
    native.call("nxs_census_device", g.ptr(d_image), w, h, g.ptr(d_codes), g.stream())
    return g.host(d_codes).view(np.uint64)


@pytest.mark.parametrize("size", [(64, 48), (97, 31), (9, 7), (364, 272)])
def test_census_codes_are_bit_exact(native, oracle, size):
    w, h = size
    image = oracle.noise(w, h, 3)
    assert (census_gpu(native, image) == oracle.census(image)).all()


def test_census_bit_order_known_answer(native):
    image = np.full((7, 9), 100, np.uint8)
    image[1, 7] = 98
    assert int(census_gpu(native, image)[3, 4]) == 1 << 14


@pytest.mark.parametrize("size,disparities", [((64, 48), 64), ((97, 31), 128), ((70, 9), 96),
                                              ((40, 20), 256), ((33, 12), 192)])
def test_costs_are_bit_exact(native, oracle, size, disparities):
    w, h = size
    left, right = oracle.noise(w, h, 1), oracle.noise(w, h, 2)
    lc, rc = oracle.census(left), oracle.census(right)
    d_l, d_r = g.dev(lc.view(np.int64)), g.dev(rc.view(np.int64))
    d_costs = g.empty((h, w, disparities), g.torch().uint8)
    native.call("nxs_costs_device", g.ptr(d_l), g.ptr(d_r), w, h, disparities, g.ptr(d_costs),
                g.stream())
    assert (g.host(d_costs).astype(np.int32) == oracle.costs(lc, rc, disparities)).all()


def aggregate_gpu(native, ctx, costs, paths, p1, p2):
    h, w, d = costs.shape
    d_costs = g.dev(costs.astype(np.uint8))
    d_sums = g.empty((h, w, d), g.torch().int16)
    native.call("nxs_aggregate_device", ctx.handle, g.ptr(d_costs), w, h, d, paths, p1, p2,
                g.ptr(d_sums), g.stream())
    return g.host(d_sums).view(np.uint16).astype(np.int32)


@pytest.mark.parametrize("size,disparities,paths", [((64, 48), 64, 8), ((64, 48), 64, 3),
                                                    ((97, 31), 128, 8), ((97, 31), 128, 3),
                                                    ((50, 40), 96, 8), ((41, 23), 192, 8),
                                                    ((37, 29), 256, 8)])
def test_aggregated_costs_are_bit_exact(native, ctx, oracle, size, disparities, paths):
    w, h = size
    left, right = oracle.scene(w, h, 7)
    costs = oracle.costs(oracle.census(left), oracle.census(right), disparities)
    want = oracle.aggregate(costs, paths, 8, 64)
    assert (aggregate_gpu(native, ctx, costs, paths, 8, 64) == want).all()


@pytest.mark.parametrize("p1,p2", [(0, 1), (4, 40), (78, 79), (10, 79)])
def test_aggregation_at_extreme_penalties(native, ctx, oracle, p1, p2):
    rng = np.random.default_rng(p1 * 100 + p2)
    costs = rng.integers(0, 49, size=(19, 45, 64)).astype(np.int32)
    want = oracle.aggregate(costs, 8, p1, p2)
    assert (aggregate_gpu(native, ctx, costs, 8, p1, p2) == want).all()


def select_gpu(native, sums, uniqueness):
    h, w, d = sums.shape
    d_sums = g.dev(sums.astype(np.uint16).view(np.int16))
    d_disp = g.empty((h, w), g.torch().float32)
    d_keys = g.empty((h, w), g.torch().int32)
    native.call("nxs_select_device", g.ptr(d_sums), w, h, d, uniqueness, g.ptr(d_disp),
                g.ptr(d_keys), g.stream())
    return g.host(d_disp), g.host(d_keys).view(np.uint32)


@pytest.mark.parametrize("disparities", [64, 128, 96, 256])
def test_selection_on_random_and_tied_sums(native, oracle, disparities):
    # select.rs:207-226: spreads that tie often and costs near the maximum.
    rng = np.random.default_rng(disparities)
    for spread in (3, 20, 1016):
        sums = rng.integers(0, spread, size=(3, 90, disparities)).astype(np.int32)
        for uniqueness in (1.0, 1.0526316, 1.2):
            want_d, want_k = oracle.select(sums, uniqueness)
            got_d, got_k = select_gpu(native, sums, uniqueness)
            assert g.same_bits(got_d, want_d) and (got_k == want_k).all()


def test_consistency_and_median(native, oracle):
    rng = np.random.default_rng(8)
    w, h = 90, 12
    keys = np.full((h, w), 0xFFFFFFFF, np.uint32)
    disparity = np.full((h, w), -1.0, np.float32)
    for y in range(h):
        for x in range(w):
            if rng.integers(5):
                winner = int(rng.integers(min(x + 1, 64)))
                keys[y, x] = (int(rng.integers(4)) << 16) | winner
                disparity[y, x] = max(winner + [0.0, 0.3, -0.4, 0.5][rng.integers(4)], 0.0)
    d_disp, d_keys = g.dev(disparity), g.dev(keys.view(np.int32))
    d_out = g.empty((h, w), g.torch().float32)
    native.call("nxs_consistency_device", g.ptr(d_disp), g.ptr(d_keys), w, h, g.ptr(d_out),
                g.stream())
    checked = g.host(d_out)
    assert g.same_bits(checked, oracle.consistency(disparity, keys, 64))
    d_med = g.empty((h, w), g.torch().float32)
    native.call("nxs_median3_device", g.ptr(d_out), w, h, 0, g.ptr(d_med), g.stream())
    assert g.same_bits(g.host(d_med), oracle.median3(checked))


CASES = [((64, 48), 64, 3), ((64, 48), 64, 8), ((64, 48), 128, 3), ((64, 48), 128, 8),
         ((97, 31), 64, 3), ((97, 31), 64, 8), ((97, 31), 128, 3), ((97, 31), 128, 8),
         # the widest image the reference takes (4096) at its least height (7), and the
         # narrowest (9) at a height of 4096: scan lines of 4096 steps along rows, and
         # along columns, in the path kernel's blocks of eight
         ((4096, 7), 64, 8), ((4096, 9), 128, 8), ((9, 4096), 64, 8)]


@pytest.mark.parametrize("size,disparities,paths", CASES)
def test_sgm_matches_the_oracle_on_scenes_and_noise(ctx, oracle, size, disparities, paths):
    w, h = size
    for left, right in (oracle.scene(w, h, 7), (oracle.noise(w, h, 1), oracle.noise(w, h, 2))):
        want = oracle.sgm(left, right, disparities, paths)
        got = ctx.sgm(left, right, disparities=disparities, paths=paths)
        assert g.same_bits(got, want)


@pytest.mark.parametrize("p1,p2,uniqueness", [(0, 1, 1.0), (4, 40, 1.2), (78, 79, 2.5),
                                              (10, 79, 1.0526316)])
def test_sgm_other_penalties_and_uniqueness(ctx, oracle, p1, p2, uniqueness):
    left, right = oracle.scene(80, 40, 3)
    for paths in (3, 8):
        want = oracle.sgm(left, right, 64, paths, p1, p2, uniqueness)
        got = ctx.sgm(left, right, disparities=64, paths=paths, p1=p1, p2=p2,
                      uniqueness=uniqueness)
        assert g.same_bits(got, want)


@pytest.mark.parametrize("disparities", [96, 192, 256])
def test_sgm_beyond_the_reference_disparities(ctx, oracle, disparities):
    # D = 96, 192, 256 are refused by the reference; the oracle's restatement
    # is D-generic, so parity holds against it (unpinned by the reference).
    left, right = oracle.scene(300, 40, 5)
    want = oracle.sgm(left, right, disparities, 8)
    assert g.same_bits(ctx.sgm(left, right, disparities=disparities, paths=8), want)


def test_sgm_at_364x272_64_disparities(ctx, oracle):
    from nx_stereo_b200 import scene

    left, right = scene.rectified_pair(364, 272, seed=1, rectangles=6, max_disparity=56)
    want = oracle.fast_sgm(left, right, 64, 8)
    assert g.same_bits(ctx.sgm(left, right, disparities=64, paths=8), want)


def test_sgm_stage_mask(ctx, oracle):
    image = oracle.noise(64, 48, 4)
    want = oracle.disparity_stage(image, image)
    assert g.same_bits(ctx.sgm(image, image, stage_mask=True), want)


def test_sgm_resizes_between_pairs(ctx, oracle):
    # lib.rs:615-628
    for w, h in [(96, 64), (64, 48), (96, 64)]:
        left, right = oracle.scene(w, h, 5)
        assert g.same_bits(ctx.sgm(left, right), oracle.sgm(left, right))


def test_sgm_recovers_a_shifted_scene(ctx, oracle):
    w, h = 96, 64
    left, right = oracle.scene(w, h, 11)
    d = ctx.sgm(left, right)
    x, y = 60, 20
    u = (x - 4.0 - 6.0 * y / h) / (1.0 + 30.0 / w)
    assert abs(d[y, x] - (x - u)) < 1.0


def test_sgm_device_entry_on_torch_buffers(native, ctx, oracle):
    left, right = oracle.scene(128, 64, 2)
    d_l, d_r = g.dev(left), g.dev(right)
    d_out = g.empty((64, 128), g.torch().float32)
    ctx.sgm_device(g.ptr(d_l), g.ptr(d_r), 128, 64, g.ptr(d_out), g.stream(), disparities=128)
    assert g.same_bits(g.host(d_out), oracle.sgm(left, right, 128, 8))


def test_refusals(ctx, native):
    image = np.zeros((48, 64), np.uint8)
    for settings in [dict(disparities=80), dict(paths=4), dict(p1=64, p2=64), dict(p2=80),
                     dict(uniqueness=0.9), dict(uniqueness=float("nan"))]:
        with pytest.raises(native.NativeError):
            ctx.sgm(image, image, **settings)
    with pytest.raises(native.NativeError):
        ctx.sgm(np.zeros((48, 8), np.uint8), np.zeros((48, 8), np.uint8))
