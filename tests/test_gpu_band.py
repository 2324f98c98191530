"""The coarse-to-fine search on the GPU (csrc/band.cu) against the reference
itself (tests/golden/reference_band.npz: the reference's own band shaders
run on the CPU) and against the oracle on fresh seeded cases: sgm_band/4 at
every band width, path count and census window, the whole coarse-to-fine
chain (its band bases too) through the device and host entry points, edge
sizes, and the size-independent properties the reference documents (a full
band from zero is the full search; a pixel without a base is never matched;
no match leaves the right image)."""
import numpy as np
import pytest

from tests import gpu_util as g
from tests.test_band_oracle import CASES, WINDOW_NAMES, bits

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from nx_stereo_b200 import native

    c = native.Context(0)
    yield c
    c.close()


def band_gpu(ctx, left, right, base, disparities=128, **settings):
    h, w = left.shape
    d_l, d_r, d_b = g.dev(left), g.dev(right), g.dev(np.ascontiguousarray(base, np.int32))
    out = g.empty((h, w), g.torch().float32)
    ctx.sgm_band_device(g.ptr(d_l), g.ptr(d_r), g.ptr(d_b), w, h, g.ptr(out), stream=g.stream(),
                        disparities=disparities, **settings)
    return g.host(out)


def coarse_to_fine_gpu(ctx, left, right, **settings):
    h, w = left.shape
    d_l, d_r = g.dev(left), g.dev(right)
    out = g.empty((h, w), g.torch().float32)
    base = g.empty((h, w), g.torch().int32)
    ctx.sgm_coarse_to_fine_device(g.ptr(d_l), g.ptr(d_r), w, h, g.ptr(out), g.ptr(base),
                                  stream=g.stream(), **settings)
    return g.host(out), g.host(base)


@pytest.mark.parametrize("name", sorted(CASES))
def test_the_cuda_band_search_equals_the_reference(ctx, name):
    case = CASES[name]
    s = [int(v) for v in case["settings"]]
    band, paths, p1, p2, window = s[:5]
    settings = dict(paths=paths, p1=p1, p2=p2, uniqueness=float(case["uniqueness"]), band=band,
                    census=WINDOW_NAMES[window])
    if len(s) > 5:
        got, base = coarse_to_fine_gpu(ctx, case["left"], case["right"], coarse_paths=s[5],
                                       margin=s[6], **settings)
        assert np.array_equal(base, case["base"])
    else:
        got = band_gpu(ctx, case["left"], case["right"], case["base"], **settings)
    assert np.array_equal(bits(got), bits(case["disparity"]))


def test_the_host_entry_point_equals_the_reference(ctx):
    case = CASES["c2f_scene_728x544_b16_p8"]
    got = ctx.sgm_coarse_to_fine(case["left"], case["right"], band=16, paths=8)
    assert np.array_equal(bits(got), bits(case["disparity"]))
    assert (got > 0).mean() > 0.85


@pytest.mark.parametrize("band", [8, 16, 32, 64])
@pytest.mark.parametrize("census", ["sparse_9x7", "dense_9x5", "dense_9x5_blend"])
def test_band_search_against_the_oracle(ctx, oracle, band, census):
    rng = np.random.default_rng(band + len(census))
    for w, h, paths in ((131, 29, 8), (9, 7, 3), (300, 17, 8)):
        left, right = oracle.scene(w, h, w + band)
        base = rng.integers(-1, 129 - band, (h, w)).astype(np.int32)
        base[:, :w // 3] = np.clip(base[:, :w // 3] // 8, 0, 128 - band)  # runs of alike bases
        p2 = int(rng.integers(1, 80))
        p1 = int(rng.integers(0, p2))
        want = oracle.sgm_band(left, right, base, 128, paths, band, census, p1, p2, 1.03)
        got = band_gpu(ctx, left, right, base, paths=paths, band=band, census=census, p1=p1,
                       p2=p2, uniqueness=1.03)
        assert np.array_equal(bits(got), bits(want)), (w, h, paths)


@pytest.mark.parametrize("w,h,band,coarse_paths", [
    (364, 272, 16, 8), (364, 272, 32, 3), (364, 272, 8, 8), (364, 272, 64, 8),
    (1280, 720, 16, 8), (4096, 14, 16, 8), (4096, 14, 64, 3), (18, 14, 8, 8), (18, 14, 64, 8)])
def test_coarse_to_fine_against_the_oracle(ctx, oracle, w, h, band, coarse_paths):
    from nx_stereo_b200 import scene

    left, right = scene.rectified_pair(w, h, seed=band + w, rectangles=6,
                                       max_disparity=min(120, max(5, w - 2)))
    want, want_base = oracle.sgm_coarse_to_fine(left, right, 8, coarse_paths, band, 4,
                                                with_base=True)
    got, base = coarse_to_fine_gpu(ctx, left, right, paths=8, coarse_paths=coarse_paths,
                                   band=band)
    assert np.array_equal(base, want_base)
    assert np.array_equal(bits(got), bits(want))


def test_full_band_from_zero_is_the_full_search_and_no_base_no_match(ctx, oracle):
    left, right = oracle.scene(97, 31, 7)
    zero = np.zeros((31, 97), np.int32)
    assert np.array_equal(bits(band_gpu(ctx, left, right, zero, disparities=64, band=64)),
                          bits(ctx.sgm(left, right, disparities=64)))
    none = np.full((31, 97), -1, np.int32)
    assert (band_gpu(ctx, left, right, none, band=16) == -1.0).all()


def test_the_stage_mask_and_refusals(ctx, oracle):
    from nx_stereo_b200 import native, scene

    left, right = scene.rectified_pair(128, 64, seed=3)
    masked, _ = coarse_to_fine_gpu(ctx, left, right, stage_mask=True)
    plain = oracle.sgm_coarse_to_fine(left, right)
    assert np.array_equal(bits(masked), bits(np.where(plain > 0, plain, np.float32(-1.0))))
    with pytest.raises(native.NativeError) as refused:
        ctx.sgm_coarse_to_fine(left[:, :127], right[:, :127])
    assert refused.value.status == native.BAD_ARGUMENT


def test_a_segment_runs_the_coarse_to_fine_search(oracle):
    """Stage.Disparity with search "coarse_to_fine" pinned to the native
    matcher, then SpeckleFilter, through CudaSegment: each pair equals the
    oracle's coarse-to-fine search with Stage.Disparity's mask, despeckled;
    pairs in flight on the segment's two lanes change nothing."""
    from nx_stereo_b200 import scene, segment, stage

    w, h = 364, 272
    geometry = segment.standard_geometry(w, h)
    status, members = segment.members(
        [(stage.Disparity, {"search": "coarse_to_fine", "num_disparities": 128,
                            "matcher": "native", "band": 16, "coarse_paths": 3}),
         stage.SpeckleFilter], geometry)
    assert status == "ok", members
    status, seg = segment.CudaSegment.build(members, geometry)
    assert status == "ok", seg
    pairs = [scene.rectified_pair(w, h, seed=60 + k, max_disparity=120) for k in range(5)]
    sent = []
    for left, right in pairs:
        status, request = segment.CudaSegment.send_request({"left": left, "right": right}, seg)
        assert status == "ok"
        sent.append(request)
    for (left, right), request in zip(pairs, sent):
        reply = segment.CudaSegment.await_(request, seg, 60000)
        assert reply[0] == "ok", reply
        d = oracle.sgm_coarse_to_fine(left, right, 8, 3, 16, 4)
        masked = np.where(d > 0, d, np.float32(-1.0)).astype(np.float32)
        want = oracle.despeckle(masked, 12, 1.0, 3)
        assert np.array_equal(bits(reply[1]["disparity"]), bits(want))
    seg.release()
