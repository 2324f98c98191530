"""nxs_port on the GPU: the records NxStereo.NativeSegment sends (configure,
then runs sent before their replies are read, as the Matcher pipelines
them) come back as the stereo_match Port replies, each run's outputs equal to
the same segment run through CudaSegment; and the Port's refusals
(main.rs:153-180): an unknown kind, a run of a segment not configured or
released."""
import numpy as np
import pytest

from nx_stereo_b200 import build, segment, stage
from tests import port_client as pc

pytestmark = pytest.mark.gpu


@pytest.fixture
def port():
    build.build()
    p = pc.Port(build.PORT)
    yield p
    assert p.close() == 0


def test_a_pipelined_segment_through_the_port_equals_cuda_segment(port):
    from nx_stereo_b200 import scene

    w, h = 364, 272
    geometry = segment.standard_geometry(w, h)
    status, members = segment.members(
        [stage.Rectification, (stage.Disparity, {"num_disparities": 64}), stage.SpeckleFilter,
         stage.TemporalFilter, stage.Depth, (stage.PointCloud, {"decimation": 4}), stage.Quality],
        geometry)
    assert status == "ok", members
    status, seg = segment.CudaSegment.build(members, geometry)
    assert status == "ok"
    config = [(kind, settings) for kind, settings in segment._configuration(seg)]
    port.send(pc.configure_record(11, geometry, config))
    rig = scene.rig(w, h)
    frames = [scene.raw_frames(*scene.rectified_pair(w, h, seed=90, frame=k, drift=2.0), rig)
              for k in range(4)]
    for left, right in frames:  # all sent before any reply is read
        port.send(pc.run_record(11, seg.inputs, [("left_frame", left), ("right_frame", right)]))
    assert port.receive() == b"\x07"
    for left, right in frames:
        times, got = pc.decode_outputs(port.receive())
        assert len(times) == len(members)
        status, want, seg = segment.run(segment.CudaSegment,
                                        {"left_frame": left, "right_frame": right}, seg, 60000)
        assert status == "ok"
        for key, value in got.items():
            expected = np.asarray(want[key])
            assert value.shape == expected.shape, key
            assert value.tobytes() == expected.astype(value.dtype).tobytes(), key
    seg.release()


def test_the_ports_refusals(port):
    geometry = {"width": 64, "height": 48, "frame_width": 64, "frame_height": 48}
    port.send(pc.configure_record(3, geometry, [("median_filter", {"kernel_size": 5.0})]))
    reply = port.receive()
    assert reply[:1] == b"\x09" and b"median_filter" in reply
    left = np.zeros((48, 64), np.uint8)
    port.send(pc.run_record(3, [{}], [("disparity", left.astype(np.float32))]))
    assert port.receive() == b"\x09segment 3 is not configured"
    port.send(pc.configure_record(4, geometry, [("depth", {})]))
    assert port.receive() == b"\x07"
    disparity = np.full((48, 64), 8.0, np.float32)
    port.send(pc.run_record(4, [{"focal_length_px": 100.0, "baseline_m": 0.1}],
                            [("disparity", disparity)]))
    times, outputs = pc.decode_outputs(port.receive())
    assert (outputs["depth_mm"] == 1250).all()
    port.send(pc.release_record(4))
    port.send(pc.run_record(4, [{"focal_length_px": 100.0, "baseline_m": 0.1}],
                            [("disparity", disparity)]))
    assert port.receive() == b"\x09segment 4 is not configured"
