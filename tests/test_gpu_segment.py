"""CudaSegment and the C ABI's segment protocol on the GPU: the reference's
stateful pipeline test (test/nx_stereo/stage/stateful_pipeline_test.exs),
full pipelines against the oracle's chain, pairs in flight, refusals, bad
runs, timing and release."""
import time

import numpy as np
import pytest

from tests import gpu_util as g

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def seg_mod():
    from nx_stereo_b200 import native, segment

    native.load()
    return segment


def run(seg_mod, segment_, entries):
    result = seg_mod.run(seg_mod.CudaSegment, entries, segment_, 60000)
    assert result[0] == "ok", result
    return result[1], result[2]


# ---------------------------------------------------------------- the reference's stateful test
GEOMETRY = {"width": 4, "height": 4, "frame_width": 4, "frame_height": 4,
            "focal_length_px": 64.0, "baseline_m": 0.125, "principal_point": (1.5, 1.5)}


def _stateful_stages(stage):
    return [(stage.SpeckleFilter, {"min_support": 0}), stage.Quality,
            (stage.TemporalFilter, {"alpha": 0.5, "delta": 2.0, "hold": 2}), stage.Depth,
            (stage.PointCloud, {"decimation": 1})]


def _assert_depth(output, disparity, focal_length):
    assert output["disparity"].tolist() == [[disparity] * 4] * 4
    assert output["depth_mm"].dtype == np.uint16 and output["cloud_points"].dtype == np.int32
    assert output["cloud_grid"].shape == (4, 4, 3) and "depth_m" not in output
    if disparity > 0:
        depth = focal_length * 0.125 / disparity
        assert output["depth_mm"].tolist() == [[round(depth * 1000)] * 4] * 4
        assert int(output["cloud_points"]) == 16
        for index, (x, y, z) in enumerate(output["cloud_grid"].reshape(16, 3)):
            assert abs(z - depth) < 1e-6
            assert abs(x - (index % 4 - 1.5) * depth / focal_length) < 1e-6
            assert abs(y - (index // 4 - 1.5) * depth / focal_length) < 1e-6
    else:
        assert (output["depth_mm"] == 0).all() and int(output["cloud_points"]) == 0
        assert np.isnan(output["cloud_grid"]).all()


def test_stateful_pipeline_keeps_history_through_updates_and_reload(seg_mod):
    from nx_stereo_b200 import stage

    status, members = seg_mod.members(_stateful_stages(stage), GEOMETRY)
    assert status == "ok"
    status, segment_ = seg_mod.CudaSegment.build(members, GEOMETRY)
    assert status == "ok"
    sequence = [(10.0, 10.0, 0.0), (12.0, 11.0, 2.0), (12.0, 11.5, 0.0), (-1.0, 11.5, 0.0),
                (-1.0, 11.5, 0.0), (-1.0, -1.0, 0.0), (50.0, 50.0, 0.0)]

    def step(segment_, current):
        entry = np.full((4, 4), current, np.float32)
        output, segment_ = run(seg_mod, segment_, {"disparity": entry})
        assert (entry == current).all()
        return output, segment_

    for current, filtered, jitter in sequence:
        output, segment_ = step(segment_, current)
        _assert_depth(output, filtered, 64.0)
        stats = stage.disparity_stats(output["quality_sums"], 16)
        assert stats["mean_px"] == max(current, 0.0)
        assert stats["matched"] == (1.0 if current > 0 else 0.0)
        assert stats["spread_px"] == 0.0 and stats["jitter_px"] == jitter
    _, state = stage.TemporalFilter.init({"alpha": 1.0, "delta": 2.0, "hold": 0}, GEOMETRY)
    segment_ = seg_mod.CudaSegment.put_member_state(segment_, 2, state)
    output, segment_ = step(segment_, 51.0)
    _assert_depth(output, 51.0, 64.0)
    assert stage.disparity_stats(output["quality_sums"], 16)["jitter_px"] == 1.0
    output, segment_ = step(segment_, -1.0)
    _assert_depth(output, -1.0, 64.0)
    geometry = dict(GEOMETRY, focal_length_px=128.0)
    _, members = seg_mod.members(_stateful_stages(stage), geometry)
    segment_ = seg_mod.CudaSegment.reload(segment_, members, geometry)
    output, segment_ = step(segment_, 12.0)
    _assert_depth(output, 12.0, 128.0)
    assert stage.disparity_stats(output["quality_sums"], 16)["jitter_px"] == 0.0
    times = seg_mod.CudaSegment.member_times(segment_)
    assert [name for name, _ in times] == ["SpeckleFilter", "Quality", "TemporalFilter", "Depth",
                                           "PointCloud"]
    assert all(ns >= 0 for _, ns in times)
    segment_.release()


def test_disparity_entries_in_either_output_layout(seg_mod, oracle):
    """A disparity passed in: TemporalFilter -> Depth also returns it (the entry's
    buffer is an output, so each output comes down on its own); Depth ->
    PointCloud does not (one packed download, and the pairs, sent together,
    compute on two streams). Each against the oracle, pair by pair."""
    from nx_stereo_b200 import stage

    w, h = 40, 24
    geometry = dict(GEOMETRY, width=w, height=h, frame_width=w, frame_height=h,
                    principal_point=(19.5, 11.5))
    rng = np.random.default_rng(5)
    maps = [np.where(rng.random((h, w)) < 0.2, -1.0, rng.uniform(1.0, 60.0, (h, w)))
            .astype(np.float32) for _ in range(5)]
    _, members = seg_mod.members([stage.TemporalFilter, stage.Depth], geometry)
    _, temporal_segment = seg_mod.CudaSegment.build(members, geometry)
    previous, missed = np.full((h, w), -1.0, np.float32), np.zeros((h, w), np.float32)
    for current in maps:
        output, temporal_segment = run(seg_mod, temporal_segment, {"disparity": current})
        want, previous, missed = oracle.temporal(current, previous, missed)
        assert g.same_bits(output["disparity"], want)
        assert (output["depth_mm"] == oracle.depth(want, 64.0, 0.125)[0]).all()
    temporal_segment.release()

    _, members = seg_mod.members([stage.Depth, (stage.PointCloud, {"decimation": 2})], geometry)
    _, cloud_segment = seg_mod.CudaSegment.build(members, geometry)
    sent = []
    for current in maps:
        status, request = seg_mod.CudaSegment.send_request({"disparity": current}, cloud_segment)
        assert status == "ok"
        sent.append(request)
    for current, request in zip(maps, sent):
        reply = seg_mod.CudaSegment.await_(request, cloud_segment, 60000)
        assert reply[0] == "ok", reply
        depth_mm, depth_m = oracle.depth(current, 64.0, 0.125)
        grid, kept = oracle.cloud(depth_m, 2, 64.0, 19.5, 11.5)
        assert (reply[1]["depth_mm"] == depth_mm).all()
        assert int(reply[1]["cloud_points"]) == kept
        got, empty = reply[1]["cloud_grid"], np.isnan(grid)
        assert (np.isnan(got) == empty).all() and g.same_bits(got[~empty], grid[~empty])
    cloud_segment.release()


# ---------------------------------------------------------------- full pipelines vs the oracle
def _oracle_chain(oracle, geometry, frames, disparities, paths, temporal=None, quality=None,
                  fast=False):
    h, w = geometry["height"], geometry["width"]
    images = [oracle.rectify(f, oracle.make_camera(c["k"], c["d"], c["inverse_pr"]), (h, w))
              for f, c in zip(frames, (geometry["left_camera"], geometry["right_camera"]))]
    if fast:  # the optimised formulation, then Stage.Disparity's mask (disparity.ex:162)
        d = oracle.fast_sgm(images[0], images[1], disparities, paths)
        d = np.where(d > 0, d, np.float32(-1.0)).astype(np.float32)
    else:
        d = oracle.disparity_stage(images[0], images[1], disparities, paths)
    d = oracle.despeckle(d, 12, 1.0, 3)
    out = {"left": images[0], "right": images[1]}
    if temporal is not None:
        d, temporal["previous"], temporal["missed"] = oracle.temporal(
            d, temporal["previous"], temporal["missed"], 0.4, 2.0, 2.0, 255.0)
    out["disparity"] = d
    mm, m = oracle.depth(d, geometry["focal_length_px"], geometry["baseline_m"])
    out["depth_mm"], out["depth_m"] = mm, m
    if quality is not None:
        out["quality_sums"], quality["previous"] = oracle.quality(d, quality["previous"])
    return out


@pytest.mark.parametrize("w,h", [(728, 544), (1280, 720)])
def test_serving_chain_over_several_pairs_matches_the_oracle(seg_mod, oracle, w, h):
    # Rectification -> Disparity(128) -> SpeckleFilter -> TemporalFilter -> Depth -> Quality,
    # the per-stream chain of the serving workload at both of its stream sizes, on
    # a scene whose surfaces drift from pair to pair, as the serving workload's do.
    from nx_stereo_b200 import scene, stage

    geometry = seg_mod.standard_geometry(w, h)
    status, members = seg_mod.members(
        [stage.Rectification, (stage.Disparity, {"num_disparities": 128}), stage.SpeckleFilter,
         stage.TemporalFilter, stage.Depth, stage.Quality], geometry)
    assert status == "ok"
    _, segment_ = seg_mod.CudaSegment.build(members, geometry)
    rig = scene.rig(w, h)
    temporal = {"previous": np.full((h, w), -1.0, np.float32), "missed": np.zeros((h, w), np.float32)}
    quality = {"previous": np.full((h, w), -1.0, np.float32)}
    for k in range(3):
        left, right = scene.rectified_pair(w, h, seed=40, rectangles=8, max_disparity=120,
                                           frame=k, drift=2.0)
        frames = scene.raw_frames(left, right, rig)
        output, segment_ = run(seg_mod, segment_, {"left_frame": frames[0],
                                                   "right_frame": frames[1]})
        want = _oracle_chain(oracle, geometry, frames, 128, 8, temporal, quality,
                             fast=w > 728)
        for name in ("left", "right", "depth_mm"):
            assert (output[name] == want[name]).all(), name
        assert g.same_bits(output["disparity"], want["disparity"])
        assert np.allclose(output["quality_sums"], want["quality_sums"], rtol=1e-5, atol=0)
    segment_.release()


def test_pairs_in_flight_equal_pairs_sent_alone(seg_mod, oracle):
    # Continuous sending: more pairs than slots at once, each result the same as alone.
    from nx_stereo_b200 import scene, stage

    w, h = 364, 272
    geometry = seg_mod.standard_geometry(w, h)
    stages = [(stage.Disparity, {"num_disparities": 64}), stage.SpeckleFilter, stage.Depth,
              (stage.PointCloud, {"decimation": 4})]
    _, members = seg_mod.members(stages, geometry)
    _, segment_ = seg_mod.CudaSegment.build(members, geometry)
    pairs = [scene.rectified_pair(w, h, seed=70 + k, max_disparity=56) for k in range(7)]
    sent = []
    for left, right in pairs:
        status, request = seg_mod.CudaSegment.send_request({"left": left, "right": right},
                                                           segment_)
        assert status == "ok"
        sent.append(request)
    together = []
    for request in sent:
        reply = seg_mod.CudaSegment.await_(request, segment_, 60000)
        assert reply[0] == "ok", reply
        together.append({k: np.array(v) for k, v in reply[1].items()})
    # These stages carry nothing, so neighbouring pairs compute on two streams at
    # once; their replies still complete in the order sent.
    stamps = [request.done_ns() for request in sent]
    assert all(stamps) and stamps == sorted(stamps)
    for (left, right), got in zip(pairs, together):
        _, alone_segment = seg_mod.CudaSegment.build(members, geometry)
        alone, _ = run(seg_mod, alone_segment, {"left": left, "right": right})
        for name in ("disparity", "depth_mm", "cloud_points", "cloud_grid"):
            assert np.asarray(got[name]).tobytes() == np.asarray(alone[name]).tobytes(), name
        want = oracle.despeckle(oracle.disparity_stage(left, right, 64, 8), 12, 1.0, 3)
        assert g.same_bits(got["disparity"], want)
        alone_segment.release()
    segment_.release()


# ---------------------------------------------------------------- the C ABI's refusals
@pytest.fixture(scope="module")
def ctx():
    from nx_stereo_b200 import native

    c = native.Context(0)
    yield c
    c.close()


def _refusal(ctx, members, geometry=(64, 48, 64, 48)):
    from nx_stereo_b200 import native

    with pytest.raises(native.NativeError) as error:
        ctx.configure(91, geometry, members)
    assert error.value.status == native.REFUSED
    return error.value.message


def test_configurations_the_segment_refuses(ctx):
    # native/stereo_match/src/segment.rs:242-333
    assert _refusal(ctx, [("sharpness", {})]) == "no native implementation of sharpness"
    assert _refusal(ctx, [("disparity", {"num_disparities": 64, "paths": 8, "zoom": 1})]) == \
        "disparity has no setting zoom"
    assert _refusal(ctx, [("disparity", {"num_disparities": 80, "paths": 8})]).startswith(
        "disparity num_disparities must be one of")
    assert _refusal(ctx, [("disparity", {"paths": 8})]) == \
        "disparity needs its num_disparities setting"
    assert _refusal(ctx, [("rectification", {})], (64, 48, 32, 48)).startswith(
        "rectification only shrinks")
    assert _refusal(ctx, [("point_cloud", {"decimation": 4, "min_depth_m": 0.05,
                                           "max_depth_m": 20.0})]) == \
        "no stage before it provides depth_m, and a segment cannot take it as an entry"
    assert _refusal(ctx, [("depth", {}), ("point_cloud", {"decimation": 49, "min_depth_m": 0.05,
                                                         "max_depth_m": 20.0})]).startswith(
        "point_cloud decimation must be an integer from 1 to 48, got 49")


def test_runs_the_segment_cannot_serve(ctx):
    from nx_stereo_b200 import native

    ctx.configure(92, (64, 48, 64, 48), [("disparity", {"num_disparities": 64, "paths": 8})])
    image = np.zeros((48, 64), np.uint8)
    good = {"p1": 8.0, "p2": 64.0, "uniqueness": 1.05}
    cases = [({"p2": 64.0, "uniqueness": 1.05}, "no p1 among the stage's inputs"),
             (dict(good, p1=1.5), "p1 must be an integer from 0 to 255, got 1.5"),
             (dict(good, p1=64.0), "expected 0 <= p1 < p2 <= 79, got 64 and 64"),
             (dict(good, uniqueness=[1.0, 2.0]), "uniqueness has 2 values, expected 1")]
    for params, message in cases:
        with pytest.raises(native.NativeError) as error:
            ctx.run_async(92, [params], {"left": image, "right": image})
        assert error.value.status == native.BAD_RUN and error.value.message == message
    with pytest.raises(native.NativeError) as error:
        ctx.run_async(92, [good], {"left": image})
    assert error.value.message == "missing entry right"
    with pytest.raises(native.NativeError) as error:
        ctx.run_async(92, [good], {"left": image, "right": np.zeros((48, 63), np.uint8)})
    assert error.value.status == native.BAD_RUN
    with pytest.raises(native.NativeError) as error:
        ctx.run_async(93, [good], {"left": image, "right": image})
    assert error.value.status == native.NO_SEGMENT
    request = ctx.run_async(92, [good], {"left": image, "right": image})
    assert request.wait(60000)
    assert (request.outputs()["disparity"] == -1.0).all()  # identical images: disparity 0
    ctx.release(92)
    with pytest.raises(native.NativeError):
        ctx.run_async(92, [good], {"left": image, "right": image})


def test_waits_poll_time_out_and_call_back(ctx):
    import threading

    from nx_stereo_b200 import scene

    ctx.configure(94, (728, 544, 728, 544), [("disparity", {"num_disparities": 128, "paths": 8})])
    left, right = scene.rectified_pair(728, 544, seed=3, max_disparity=120)
    done = threading.Event()
    tags = []

    def callback(user, tag):
        tags.append(tag)
        done.set()

    sent_ns = time.monotonic_ns()
    request = ctx.run_async(94, [{"p1": 8.0, "p2": 64.0, "uniqueness": 1.05}],
                            {"left": left, "right": right}, done=callback, tag=77)
    first = request.wait(0)  # may or may not be done already
    assert request.wait(60000)
    seen_ns = time.monotonic_ns()
    assert request.poll() and (first in (True, False))
    assert done.wait(10) and tags == [77]
    times = request.times_us()
    assert len(times) == 1 and times[0] > 0
    # The completion time, read from the device's timestamp of the request's done
    # event, lies between its sending and the host seeing it done (the mapping onto
    # CLOCK_MONOTONIC is good to a few microseconds), after the member's time.
    done_ns = request.done_ns()
    assert sent_ns + times[0] * 1000 - 20_000 <= done_ns <= seen_ns + 20_000
    assert request.done_ns() == done_ns
    request.free()
    ctx.release(94)
