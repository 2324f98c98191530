"""The matcher's internal disparity order: the _ordered entry points write and
read the same values as the natural-order ones (which the oracle pins), each
run of `span` disparities permuted so that bytes 4q .. 4q + 3 hold
disparities 2q, 2q + 1, 2q + span / 2 and 2q + 1 + span / 2 (a path lane's
words 2q and 2q + 1, each word k holding k and k + span / 2, interleaved);
selection from ordered volumes equals selection from natural ones bit for
bit."""
import numpy as np
import pytest

from tests import gpu_util as g

pytestmark = pytest.mark.gpu

# (dy, dx) of each path volume, in the reference's order (lib/nx_stereo.ex:566-570).
DIRECTIONS = [(0, 1), (0, -1), (1, 0), (-1, 0), (1, 1), (1, -1), (-1, 1), (-1, -1)]


def position(d, span):
    """Where natural disparity d lies in the permuted order of `span`."""
    d = np.asarray(d)
    if span == 0:
        return d
    half = span // 2
    within = d % span
    return (d // span) * span + 4 * ((within % half) // 2) + d % 2 + 2 * (within // half)


def permuted(volume, span):
    out = np.empty_like(volume)
    out[..., position(np.arange(volume.shape[-1]), span)] = volume
    return out


def test_position_is_a_permutation_and_pairs_neighbours():
    for span in (8, 16):
        p = position(np.arange(64), span)
        assert sorted(p.tolist()) == list(range(64))
        inverse = np.argsort(p)  # byte j of a run holds disparity inverse[j]
        # bytes 4q .. 4q + 3: words 2q and 2q + 1 interleaved, word k = (k, k + span / 2)
        assert inverse[:span].tolist() == [2 * (j // 4) + j % 2 + (span // 2) * ((j // 2) % 2)
                                           for j in range(span)]


@pytest.fixture(scope="module")
def native():
    from nx_stereo_b200 import native as n

    n.load()
    return n


def _codes(oracle, w, h):
    left, right = oracle.scene(w, h, 7)
    return oracle.census(left), oracle.census(right)


@pytest.mark.parametrize("span", [8, 16])
@pytest.mark.parametrize("disparities", [64, 96, 128, 256])
def test_ordered_costs(native, oracle, span, disparities):
    w, h = 70, 23
    lc, rc = _codes(oracle, w, h)
    d_l, d_r = g.dev(lc.view(np.int64)), g.dev(rc.view(np.int64))
    d_costs = g.empty((h, w, disparities), g.torch().uint8)
    native.call("nxs_costs_device_ordered", g.ptr(d_l), g.ptr(d_r), w, h, disparities, span,
                g.ptr(d_costs), g.stream())
    want = oracle.costs(lc, rc, disparities).astype(np.uint8)
    assert (g.host(d_costs) == permuted(want, span)).all()


@pytest.mark.parametrize("span", [0, 8, 16])
@pytest.mark.parametrize("disparities", [16, 64, 96, 128, 192, 256])
@pytest.mark.parametrize("w,h", [(70, 23), (9, 7), (131, 5), (300, 17), (4096, 7)])
def test_census_and_costs_in_one_launch(native, oracle, span, disparities, w, h):
    """nxs_census_costs_device_ordered forms the codes in shared memory: its
    costs equal the oracle's census then costs, at widths below, across and
    not a multiple of its 128-pixel blocks and of the census's four pixels."""
    left, right = oracle.scene(w, h, 11)
    d_left, d_right = g.dev(left), g.dev(right)
    d_costs = g.empty((h, w, disparities), g.torch().uint8)
    native.call("nxs_census_costs_device_ordered", g.ptr(d_left), g.ptr(d_right), w, h,
                disparities, span, g.ptr(d_costs), g.stream())
    want = oracle.costs(oracle.census(left), oracle.census(right), disparities).astype(np.uint8)
    assert (g.host(d_costs) == permuted(want, span)).all()


@pytest.mark.parametrize("span", [8, 16])
@pytest.mark.parametrize("disparities,paths", [(64, 8), (128, 8), (128, 3), (256, 8), (96, 8)])
def test_ordered_paths_and_selection(native, oracle, span, disparities, paths):
    torch = g.torch()
    w, h = 61, 29
    lc, rc = _codes(oracle, w, h)
    d_l, d_r = g.dev(lc.view(np.int64)), g.dev(rc.view(np.int64))
    vol = h * w * disparities
    natural = {"costs": g.empty(vol, torch.uint8), "paths": g.empty(paths * vol, torch.uint8),
               "disparity": g.empty(h * w, torch.float32), "keys": g.empty(h * w, torch.int32)}
    ordered = {k: torch.empty_like(v) for k, v in natural.items()}
    for out, sp in ((natural, 0), (ordered, span)):
        native.call("nxs_costs_device_ordered", g.ptr(d_l), g.ptr(d_r), w, h, disparities, sp,
                    g.ptr(out["costs"]), g.stream())
        native.call("nxs_paths_device_ordered", g.ptr(out["costs"]), w, h, disparities, paths, 8,
                    64, sp, g.ptr(out["paths"]), g.stream())
        native.call("nxs_select_paths_device_ordered", g.ptr(out["paths"]), w, h, disparities,
                    paths, 1.0526315789473684, sp, g.ptr(out["disparity"]), g.ptr(out["keys"]),
                    g.stream())
    n_paths = g.host(natural["paths"]).reshape(paths, h, w, disparities)
    o_paths = g.host(ordered["paths"]).reshape(paths, h, w, disparities)
    assert (o_paths == permuted(n_paths, span)).all()
    costs = oracle.costs(lc, rc, disparities)
    for p in range(paths):  # the natural volumes against the oracle
        assert (n_paths[p].astype(np.int32) == oracle.path(costs, DIRECTIONS[p], 8, 64)).all()
    assert g.same_bits(g.host(ordered["disparity"]), g.host(natural["disparity"]))
    assert (g.host(ordered["keys"]) == g.host(natural["keys"])).all()


def test_the_matchers_span(native):
    lib = native.load()
    for d in (64, 96, 128, 192, 256):
        assert lib.nxs_matcher_span(d) == (8 if lib.nxs_path_words(d) == 4 else 16)
    with pytest.raises(native.NativeError):
        native.call("nxs_costs_device_ordered", 1, 1, 8, 8, 64, 4, 1, None)
    with pytest.raises(native.NativeError):  # a span the kernels do not take
        native.call("nxs_census_costs_device_ordered", 1, 1, 8, 8, 64, 4, 1, None)
    with pytest.raises(native.NativeError):  # not a multiple of 16 disparities
        native.call("nxs_census_costs_device_ordered", 1, 1, 8, 8, 72, 16, 1, None)
