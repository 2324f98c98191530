"""A segment whose matcher runs split over two streams (each pair's census,
costs and path volumes on one, its selection onwards on the other, pairs
alternating between two scratches) gives every pair the same outputs as the
unsplit segment and as the oracle, with many pairs in flight."""
import numpy as np
import pytest

from tests import gpu_util as g

pytestmark = pytest.mark.gpu


CHAIN = "cloud"  # the stateless chain; "state": the serving chain with temporal and quality


def _stages(chain, disparities=128):
    from nx_stereo_b200 import stage

    if chain == "state":
        return [stage.Rectification, (stage.Disparity, {"num_disparities": 128}),
                stage.SpeckleFilter, stage.TemporalFilter, stage.Depth, stage.Quality]
    return [stage.Rectification, (stage.Disparity, {"num_disparities": disparities}),
            stage.SpeckleFilter, stage.Depth, (stage.PointCloud, {"decimation": 4})]


def _run(split, pairs, frames_of, w, h, chain=CHAIN, lean=None, disparities=128):
    from nx_stereo_b200 import native, segment

    native.load().nxs_set_split_lanes(1 if split else 0)
    lean_before = native.load().nxs_lean_select()
    if lean is not None:
        assert native.load().nxs_set_lean_select(lean) == 0
    try:
        geometry = segment.standard_geometry(w, h)
        status, members = segment.members(_stages(chain, disparities), geometry)
        assert status == "ok", members
        status, seg = segment.CudaSegment.build(members, geometry)
        assert status == "ok", seg
        sent = []
        for k in range(pairs):  # all sent before any is awaited
            status, request = segment.CudaSegment.send_request(frames_of(k), seg)
            assert status == "ok"
            sent.append(request)
        replies = []
        for request in sent:
            reply = segment.CudaSegment.await_(request, seg, 60000)
            assert reply[0] == "ok", reply
            replies.append({k: np.array(v) for k, v in reply[1].items()})
        seg.release()
        return replies
    finally:
        native.load().nxs_set_split_lanes(1)
        native.load().nxs_set_lean_select(lean_before)


def test_split_equals_unsplit_and_the_oracle(oracle):
    from nx_stereo_b200 import scene, segment

    w, h = 728, 544
    rig = scene.rig(w, h)
    frames = []
    for k in range(6):
        left, right = scene.rectified_pair(w, h, seed=90 + k, rectangles=6, max_disparity=120)
        frames.append(scene.raw_frames(left, right, rig))

    def frames_of(k):
        return {"left_frame": frames[k % 6][0], "right_frame": frames[k % 6][1]}

    split = _run(True, 9, frames_of, w, h)
    plain = _run(False, 9, frames_of, w, h)
    for a, b in zip(split, plain):
        assert a.keys() == b.keys()
        for key in a:
            assert a[key].tobytes() == b[key].tobytes(), key
    # the first pair against the oracle's chain
    geometry = segment.standard_geometry(w, h)
    cams = [geometry["left_camera"], geometry["right_camera"]]
    images = [oracle.rectify(f, oracle.make_camera(c["k"], c["d"], c["inverse_pr"]), (h, w))
              for f, c in zip(frames[0], cams)]
    d = oracle.fast_sgm(images[0], images[1], 128, 8)
    d = np.where(d > 0, d, np.float32(-1.0)).astype(np.float32)
    want = oracle.despeckle(d, 12, 1.0, 3)
    assert g.same_bits(split[0]["disparity"], want)


def test_split_keeps_the_state_in_order():
    """The serving chain (TemporalFilter and Quality carry state from pair to
    pair): split, its state advances on the back stream in request order, so
    every pair's outputs equal those of the segment run on one stream."""
    from nx_stereo_b200 import scene

    w, h = 364, 272
    rig = scene.rig(w, h)
    frames = []
    for k in range(5):
        left, right = scene.rectified_pair(w, h, seed=130 + k, rectangles=6, max_disparity=56)
        frames.append(scene.raw_frames(left, right, rig))

    def frames_of(k):
        return {"left_frame": frames[k % 5][0], "right_frame": frames[k % 5][1]}

    split = _run(True, 8, frames_of, w, h, chain="state")
    plain = _run(False, 8, frames_of, w, h, chain="state")
    for a, b in zip(split, plain):
        assert a.keys() == b.keys()
        for key in a:
            assert a[key].tobytes() == b[key].tobytes(), key


@pytest.mark.parametrize("lean", [0, 1, 3, 16])
def test_lean_selection_is_the_same(lean):
    """The selection a split segment runs beside the next pair's path scan, as a
    grid of `lean` blocks a SM stepping through the pixel blocks (0: one block
    for each), gives the same outputs as the segment on one stream."""
    from nx_stereo_b200 import scene

    w, h = 500, 301  # a ragged last pixel block
    rig = scene.rig(w, h)
    frames = []
    for k in range(3):
        left, right = scene.rectified_pair(w, h, seed=170 + k, rectangles=5, max_disparity=100)
        frames.append(scene.raw_frames(left, right, rig))

    def frames_of(k):
        return {"left_frame": frames[k % 3][0], "right_frame": frames[k % 3][1]}

    split = _run(True, 6, frames_of, w, h, lean=lean)
    plain = _run(False, 6, frames_of, w, h)
    for a, b in zip(split, plain):
        assert a.keys() == b.keys()
        for key in a:
            assert a[key].tobytes() == b[key].tobytes(), key


@pytest.mark.parametrize("disparities", [64, 256])
def test_lean_selection_other_lane_counts(disparities):
    """The lean selection with 4 and 16 lanes a pixel (64 and 256 disparities),
    at its default setting and with one block a SM, against the segment on one
    stream."""
    from nx_stereo_b200 import scene

    w, h = 420, 197
    rig = scene.rig(w, h)
    frames = []
    for k in range(3):
        left, right = scene.rectified_pair(w, h, seed=190 + k, rectangles=5,
                                           max_disparity=min(disparities - 8, 200))
        frames.append(scene.raw_frames(left, right, rig))

    def frames_of(k):
        return {"left_frame": frames[k % 3][0], "right_frame": frames[k % 3][1]}

    plain = _run(False, 5, frames_of, w, h, disparities=disparities)
    for lean in (None, 1):
        split = _run(True, 5, frames_of, w, h, lean=lean, disparities=disparities)
        for a, b in zip(split, plain):
            assert a.keys() == b.keys()
            for key in a:
                assert a[key].tobytes() == b[key].tobytes(), (lean, key)
